// Binary model file: a continuous LP/QP (nk_model) stored as its raw arrays so
// that a large instance loads by mapping the file instead of parsing text.
//
// The reference reads models only as text (its native JSON format and MPS,
// src/io.cpp:84-139,299,800) and its Python session hands a model to the
// library through a temporary JSON file (python/vantage/native.py:26-31); for
// an instance of 20 million nonzeros that parse dominates the time to the
// first iteration.  This format holds the same fields as the JSON model
// (A, Q, c, q, bounds, row bounds, offset) in the engine's host layout:
//
//   offset 0    header, 128 bytes, little-endian
//     char[8]   magic "NKMODEL1"
//     uint32    version (1)
//     uint32    flags (bit 0: Q present; bit 1: the source objective was
//               maximised -- c, q, Q and the offset hold its minimisation form,
//               their negation, the way the reference canonicalises a model,
//               src/io.cpp:74-80)
//     int64     m, n, nnz, qnnz
//     double    objective offset
//     uint64    payload bytes (everything after the header)
//     uint64    payload checksum (below)
//     zeros up to byte 128
//   offset 128  the arrays, each starting on a 64-byte boundary, zero padded:
//     A.ptr[m+1] (int64), A.index[nnz] (int64), A.value[nnz] (double),
//     c[n], q[n], lb[n], ub[n], rl[m], ru[m] (double),
//     and with Q: Q.ptr[n+1], Q.index[qnnz] (int64), Q.value[qnnz] (double).
//
// Infinite bounds are stored as IEEE infinities.  The checksum is FNV-1a
// (Fowler-Noll-Vo) applied to 64-bit words instead of bytes, in four
// interleaved lanes (word k goes to lane k mod 4) that are folded together at
// the end, so the loop is not one serial multiply chain.  A reader maps the
// file and points an nk_model into the mapping after checking the header, the
// file size, the checksum and the CSR structure (offsets from 0, never
// decreasing, ending at nnz; every column index inside [0, n)).
#include "nk_common.cuh"

#include <cerrno>
#include <cstring>
#include <fcntl.h>
#include <memory>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

namespace nk {
namespace {

constexpr char kMagic[8] = {'N', 'K', 'M', 'O', 'D', 'E', 'L', '1'};
constexpr uint32_t kVersion = 1;
constexpr size_t kHeaderBytes = 128;
constexpr size_t kAlign = 64;
constexpr uint64_t kFnvBasis = 14695981039346656037ull;
constexpr uint64_t kFnvPrime = 1099511628211ull;

struct Header {
    char magic[8];
    uint32_t version, flags;
    int64_t m, n, nnz, qnnz;
    double offset;
    uint64_t payload_bytes, checksum;
};
static_assert(sizeof(Header) <= kHeaderBytes, "header fits its slot");

size_t padded(size_t bytes) { return (bytes + kAlign - 1) / kAlign * kAlign; }

struct Checksum {
    uint64_t lane[4] = {kFnvBasis, kFnvBasis, kFnvBasis, kFnvBasis};
    uint64_t words = 0;
    // `bytes` is a multiple of 8 (every array is padded to 64 bytes)
    void add(const void *data, size_t bytes) {
        const unsigned char *p = static_cast<const unsigned char *>(data);
        const size_t count = bytes / 8;
        size_t k = 0;
        while (k < count && (words + k) % 4) {
            feed(p + 8 * k, (words + k) % 4);
            ++k;
        }
        for (; k + 4 <= count; k += 4) {
            uint64_t w[4];
            std::memcpy(w, p + 8 * k, 32);
            for (int l = 0; l < 4; ++l)
                lane[l] = (lane[l] ^ w[l]) * kFnvPrime;
        }
        for (; k < count; ++k)
            feed(p + 8 * k, (words + k) % 4);
        words += count;
    }
    void feed(const unsigned char *p, uint64_t l) {
        uint64_t w;
        std::memcpy(&w, p, 8);
        lane[l] = (lane[l] ^ w) * kFnvPrime;
    }
    uint64_t value() const {
        uint64_t h = kFnvBasis;
        for (uint64_t l : lane)
            h = (h ^ l) * kFnvPrime;
        return (h ^ words) * kFnvPrime;
    }
};

// The arrays of a model in file order: address, bytes.
struct Part {
    const void *data;
    size_t bytes;
};

std::vector<Part> parts_of(const nk_model &M, bool has_q) {
    const int64_t m = M.A.rows, n = M.A.cols, nnz = M.A.ptr[m];
    std::vector<Part> v = {{M.A.ptr, size_t(m + 1) * 8}, {M.A.index, size_t(nnz) * 8},
                           {M.A.value, size_t(nnz) * 8}, {M.c, size_t(n) * 8},
                           {M.q, size_t(n) * 8},         {M.lb, size_t(n) * 8},
                           {M.ub, size_t(n) * 8},        {M.rl, size_t(m) * 8},
                           {M.ru, size_t(m) * 8}};
    if (has_q) {
        const int64_t qnnz = M.Q.ptr[n];
        v.push_back({M.Q.ptr, size_t(n + 1) * 8});
        v.push_back({M.Q.index, size_t(qnnz) * 8});
        v.push_back({M.Q.value, size_t(qnnz) * 8});
    }
    return v;
}

// CSR structure: offsets start at 0, never decrease, end at `nnz`; every
// column index lies in [0, cols).
void check_structure(const int64_t *ptr, const int64_t *index, int64_t rows, int64_t cols,
                     int64_t nnz, const char *what) {
    if (ptr[0] != 0 || ptr[rows] != nnz)
        throw Error(NK_ERR_INVALID, std::string("model file: invalid ") + what + " CSR storage");
    for (int64_t i = 0; i < rows; ++i)
        if (ptr[i + 1] < ptr[i])
            throw Error(NK_ERR_INVALID, std::string("model file: invalid ") + what + " CSR offsets");
    for (int64_t k = 0; k < nnz; ++k)
        if (index[k] < 0 || index[k] >= cols)
            throw Error(NK_ERR_INVALID,
                        std::string("model file: ") + what + " column index out of range");
}

bool model_has_q(const nk_model &M) {
    return M.Q.rows > 0 && M.Q.ptr && M.Q.ptr[M.Q.rows] > 0;
}

void write_model(const char *path, const nk_model *model, bool maximise) {
    if (!path || !model)
        throw Error(NK_ERR_INVALID, "null argument");
    const nk_model &M = *model;
    const int64_t m = M.A.rows, n = M.A.cols;
    if (m < 0 || n < 0 || !M.A.ptr || !M.c || !M.lb || !M.ub || !M.rl || !M.ru)
        throw Error(NK_ERR_INVALID, "incomplete model");
    const int64_t nnz = M.A.ptr[m];
    if (nnz < 0 || (nnz > 0 && (!M.A.index || !M.A.value)))
        throw Error(NK_ERR_INVALID, "missing A entries");
    check_structure(M.A.ptr, M.A.index, m, n, nnz, "A");
    const bool has_q = model_has_q(M);
    int64_t qnnz = 0;
    if (has_q) {
        if (M.Q.rows != n || M.Q.cols != n || !M.Q.index || !M.Q.value)
            throw Error(NK_ERR_INVALID, "inconsistent Q dimensions");
        qnnz = M.Q.ptr[n];
        check_structure(M.Q.ptr, M.Q.index, n, n, qnnz, "Q");
    }
    // a model without q stores zeros
    std::vector<double> zero_q;
    nk_model W = M;
    if (!W.q) {
        zero_q.assign(size_t(n), 0.0);
        W.q = zero_q.data();
    }
    const std::vector<Part> parts = parts_of(W, has_q);

    Header h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.flags = (has_q ? 1u : 0u) | (maximise ? 2u : 0u);
    h.m = m;
    h.n = n;
    h.nnz = nnz;
    h.qnnz = qnnz;
    h.offset = M.offset;
    Checksum sum;
    static const unsigned char zeros[kAlign] = {};
    for (const Part &p : parts) {
        if (p.bytes)
            sum.add(p.data, p.bytes);
        if (padded(p.bytes) > p.bytes)
            sum.add(zeros, padded(p.bytes) - p.bytes);
        h.payload_bytes += padded(p.bytes);
    }
    h.checksum = sum.value();

    // write beside the target and rename, so a reader never maps a partial file
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f)
        throw Error(NK_ERR_INVALID, "model file: cannot create " + tmp + ": " + std::strerror(errno));
    unsigned char head[kHeaderBytes] = {};
    std::memcpy(head, &h, sizeof(h));
    bool ok = std::fwrite(head, 1, kHeaderBytes, f) == kHeaderBytes;
    for (const Part &p : parts) {
        if (!ok)
            break;
        if (p.bytes)
            ok = std::fwrite(p.data, 1, p.bytes, f) == p.bytes;
        const size_t pad = padded(p.bytes) - p.bytes;
        if (ok && pad)
            ok = std::fwrite(zeros, 1, pad, f) == pad;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok || std::rename(tmp.c_str(), path) != 0) {
        const std::string why = std::strerror(errno);
        std::remove(tmp.c_str());
        throw Error(NK_ERR_INVALID, std::string("model file: cannot write ") + path + ": " + why);
    }
}

// Points `out` into a model-file image of `bytes` bytes after checking it.
void view_model(const void *image, int64_t bytes, nk_model *out, int *maximise) {
    if (!image || !out || bytes < 0)
        throw Error(NK_ERR_INVALID, "null argument");
    if (size_t(bytes) < kHeaderBytes)
        throw Error(NK_ERR_INVALID, "model file: shorter than its header");
    if (reinterpret_cast<uintptr_t>(image) % 8)
        throw Error(NK_ERR_INVALID, "model file: image not 8-byte aligned");
    Header h;
    std::memcpy(&h, image, sizeof(h));
    if (std::memcmp(h.magic, kMagic, 8) != 0)
        throw Error(NK_ERR_INVALID, "model file: bad magic (not a model file)");
    if (h.version != kVersion)
        throw Error(NK_ERR_INVALID, "model file: unsupported version " + std::to_string(h.version));
    if (h.flags > 3)
        throw Error(NK_ERR_INVALID, "model file: unknown flags");
    // sizes bounded so that no byte count below overflows
    const int64_t limit = int64_t(1) << 40;
    if (h.m < 0 || h.n < 0 || h.nnz < 0 || h.qnnz < 0 || h.m > limit || h.n > limit ||
        h.nnz > limit || h.qnnz > limit || ((h.flags & 1) == 0 && h.qnnz != 0))
        throw Error(NK_ERR_INVALID, "model file: bad dimensions");
    const bool has_q = h.flags & 1;
    const size_t m = size_t(h.m), n = size_t(h.n), nnz = size_t(h.nnz), qnnz = size_t(h.qnnz);
    std::vector<size_t> sizes = {(m + 1) * 8, nnz * 8, nnz * 8, n * 8, n * 8,
                                 n * 8,       n * 8,   m * 8,   m * 8};
    if (has_q) {
        sizes.push_back((n + 1) * 8);
        sizes.push_back(qnnz * 8);
        sizes.push_back(qnnz * 8);
    }
    size_t payload = 0;
    for (size_t s : sizes)
        payload += padded(s);
    if (h.payload_bytes != payload || size_t(bytes) != kHeaderBytes + payload)
        throw Error(NK_ERR_INVALID, "model file: size does not match its header (truncated?)");
    const unsigned char *base = static_cast<const unsigned char *>(image) + kHeaderBytes;
    Checksum sum;
    sum.add(base, payload);
    if (sum.value() != h.checksum)
        throw Error(NK_ERR_INVALID, "model file: checksum mismatch (corrupted)");
    std::vector<const void *> at;
    size_t pos = 0;
    for (size_t s : sizes) {
        at.push_back(base + pos);
        pos += padded(s);
    }
    nk_model v{};
    v.A.rows = h.m;
    v.A.cols = h.n;
    v.A.ptr = static_cast<const int64_t *>(at[0]);
    v.A.index = static_cast<const int64_t *>(at[1]);
    v.A.value = static_cast<const double *>(at[2]);
    v.c = static_cast<const double *>(at[3]);
    v.q = static_cast<const double *>(at[4]);
    v.lb = static_cast<const double *>(at[5]);
    v.ub = static_cast<const double *>(at[6]);
    v.rl = static_cast<const double *>(at[7]);
    v.ru = static_cast<const double *>(at[8]);
    v.offset = h.offset;
    check_structure(v.A.ptr, v.A.index, h.m, h.n, h.nnz, "A");
    if (has_q) {
        v.Q.rows = v.Q.cols = h.n;
        v.Q.ptr = static_cast<const int64_t *>(at[9]);
        v.Q.index = static_cast<const int64_t *>(at[10]);
        v.Q.value = static_cast<const double *>(at[11]);
        check_structure(v.Q.ptr, v.Q.index, h.n, h.n, h.qnnz, "Q");
    }
    *out = v;
    if (maximise)
        *maximise = (h.flags & 2) ? 1 : 0;
}

} // namespace
} // namespace nk

struct nk_model_file {
    void *map = nullptr;
    size_t bytes = 0;
    ~nk_model_file() {
        if (map)
            munmap(map, bytes);
    }
};

extern "C" {
nk_status nk_model_write(const char *path, const nk_model *model, int maximise) {
    return nk::guard([&] { nk::write_model(path, model, maximise != 0); });
}

nk_status nk_model_view(const void *image, int64_t bytes, nk_model *model, int *maximise) {
    return nk::guard([&] { nk::view_model(image, bytes, model, maximise); });
}

nk_status nk_model_open(const char *path, nk_model_file **file, nk_model *model, int *maximise) {
    return nk::guard([&] {
        if (!path || !file || !model)
            throw nk::Error(NK_ERR_INVALID, "null argument");
        *file = nullptr;
        const int fd = ::open(path, O_RDONLY | O_CLOEXEC);
        if (fd < 0)
            throw nk::Error(NK_ERR_INVALID,
                            std::string("model file: cannot open ") + path + ": " + std::strerror(errno));
        struct stat st {};
        if (::fstat(fd, &st) != 0 || st.st_size <= 0) {
            ::close(fd);
            throw nk::Error(NK_ERR_INVALID, std::string("model file: empty or unreadable ") + path);
        }
        auto f = std::make_unique<nk_model_file>();
        f->bytes = size_t(st.st_size);
        void *map = ::mmap(nullptr, f->bytes, PROT_READ, MAP_PRIVATE, fd, 0);
        ::close(fd);
        if (map == MAP_FAILED)
            throw nk::Error(NK_ERR_MEMORY, std::string("model file: cannot map ") + path);
        f->map = map;
        nk::view_model(f->map, int64_t(f->bytes), model, maximise);
        *file = f.release();
    });
}

void nk_model_close(nk_model_file *file) { delete file; }
}
