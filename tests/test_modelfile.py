"""Binary model files (CPU only): the layout, the checks on reading, and parity
with the reference's own JSON reader.

The file format is restated here from its specification (header fields, 64-byte
aligned arrays, the four-lane word-wise FNV-1a checksum) and the library's
writer must produce the same bytes.  The restatement also builds files with a
valid checksum but a broken structure, which the reader must refuse.  The
reference's read_model (src/io.cpp:800-814) reading the native JSON of a model
must give exactly the arrays the model file holds."""
import ctypes as C
import json
import struct

import numpy as np
import pytest

from niryukti_b200 import engine, modelfile, serve, solver, synth
from tests.test_oracle import sparse_qp_model

MASK = (1 << 64) - 1
FNV_BASIS, FNV_PRIME = 14695981039346656037, 1099511628211


def _checksum(payload: bytes) -> int:
    words = np.frombuffer(payload, dtype="<u8").tolist()
    lanes = [FNV_BASIS] * 4
    for k, w in enumerate(words):
        lanes[k % 4] = ((lanes[k % 4] ^ w) * FNV_PRIME) & MASK
    h = FNV_BASIS
    for lane in lanes:
        h = ((h ^ lane) * FNV_PRIME) & MASK
    return ((h ^ len(words)) * FNV_PRIME) & MASK


def _pad(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 64)


def spec_file(model, maximise=False, version=1, checksum=None) -> bytes:
    """The model file as the format specifies it, built without the library."""
    m, n = model.m, model.n
    q = np.zeros(n) if model.q is None else model.q
    parts = [model.ptr, model.idx, model.val, model.c, q, model.lb, model.ub, model.rl, model.ru]
    has_q = model.qptr is not None and int(model.qptr[-1]) > 0
    if has_q:
        parts += [model.qptr, model.qidx, model.qval]
    payload = b"".join(_pad(np.ascontiguousarray(a, dtype=a.dtype.newbyteorder("<")).tobytes())
                       for a in parts)
    flags = (1 if has_q else 0) | (2 if maximise else 0)
    qnnz = int(model.qptr[-1]) if has_q else 0
    head = struct.pack("<8sIIqqqqdQQ", b"NKMODEL1", version, flags, m, n, int(model.ptr[-1]),
                       qnnz, float(model.offset), len(payload),
                       _checksum(payload) if checksum is None else checksum)
    return head.ljust(128, b"\0") + payload


def _lp():
    m = synth.random_lp(m=60, n=150, per_col=3, seed=11)
    m.lb = m.lb.copy()
    m.ub = m.ub.copy()
    m.lb[:7], m.ub[3:9] = -np.inf, np.inf  # free and one-sided columns
    m.offset = 2.5
    return m


def _same(a, b):
    for f in ("ptr", "idx", "val", "c", "q", "lb", "ub", "rl", "ru"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert (a.qptr is None) == (b.qptr is None)
    if a.qptr is not None:
        for f in ("qptr", "qidx", "qval"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert a.offset == b.offset and a.m == b.m and a.n == b.n


@pytest.mark.parametrize("make", [_lp, sparse_qp_model], ids=["lp", "qp"])
def test_round_trip(tmp_path, make):
    model = make()
    path = tmp_path / "model.nkm"
    modelfile.save(model, path)
    back = modelfile.load(path)
    _same(model, back)
    assert back.sense == 1.0 and not back.val.flags.writeable  # views of the mapping
    assert path.read_bytes() == spec_file(model)
    assert not (tmp_path / "model.nkm.tmp").exists()


def test_loaded_model_goes_through_the_library_unchanged(tmp_path):
    """The mapped arrays pass straight into nk_prepare: the prepared model is
    bit-identical to the one prepared from the in-memory arrays."""
    model = _lp()
    modelfile.save(model, tmp_path / "m.nkm")
    a = solver.prepare(model)
    b = solver.prepare(modelfile.load(tmp_path / "m.nkm"))
    assert a.keys() == b.keys()
    for k in a:
        if isinstance(a[k], np.ndarray):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert a[k] == b[k], k


def test_open_through_the_c_abi(tmp_path):
    model = sparse_qp_model()
    path = tmp_path / "qp.nkm"
    modelfile.save(model, path)
    L = C.CDLL(str(engine.LIB_PATH))
    f, v, sense = C.c_void_p(), solver.NkModel(), C.c_int(-1)
    assert L.nk_model_open(str(path).encode(), C.byref(f), C.byref(v), C.byref(sense)) == 0
    try:
        assert (v.A.rows, v.A.cols, sense.value) == (model.m, model.n, 0)
        nnz = int(model.ptr[-1])
        assert np.array_equal(np.ctypeslib.as_array(v.A.value, (nnz,)), model.val)
        assert np.array_equal(np.ctypeslib.as_array(v.Q.index, (model.qnnz,)), model.qidx)
        assert np.array_equal(np.ctypeslib.as_array(v.ru, (model.m,)), model.ru)
    finally:
        L.nk_model_close(f)
    L.nk_last_error.restype = C.c_char_p
    assert L.nk_model_open(str(tmp_path / "absent.nkm").encode(), C.byref(f), C.byref(v),
                           None) == 1
    assert b"cannot open" in L.nk_last_error()


def test_maximisation_is_recorded(tmp_path):
    d = serve.model_to_json(_lp())
    d["sense"] = "max"
    model = serve.model_from_json(json.loads(json.dumps(serve._finite(d))))
    modelfile.save(model, tmp_path / "max.nkm")
    back = modelfile.load(tmp_path / "max.nkm")
    assert back.sense == -1.0
    assert np.array_equal(back.c, model.c) and back.offset == model.offset
    assert (tmp_path / "max.nkm").read_bytes() == spec_file(model, maximise=True)


def _refused(tmp_path, data, match):
    path = tmp_path / "bad.nkm"
    path.write_bytes(data)
    with pytest.raises(engine.EngineError, match=match) as e:
        modelfile.load(path)
    assert e.value.status == "INVALID"


def test_damaged_files_are_refused(tmp_path):
    model = _lp()
    good = spec_file(model)
    flipped = bytearray(good)
    flipped[128 + 8 * 300] ^= 0x10  # one bit of the column indices
    _refused(tmp_path, bytes(flipped), "checksum mismatch")
    _refused(tmp_path, good[:-64], "size does not match")
    _refused(tmp_path, good + b"\0" * 64, "size does not match")
    _refused(tmp_path, b"XKMODEL1" + good[8:], "bad magic")
    _refused(tmp_path, spec_file(model, version=2), "unsupported version")
    _refused(tmp_path, good[:100], "shorter than its header")
    _refused(tmp_path, b"", "shorter than its header")
    _refused(tmp_path, spec_file(model, checksum=12345), "checksum mismatch")


def test_broken_structure_with_a_valid_checksum_is_refused(tmp_path):
    model = _lp()
    bad = synth.Model(**{**model.__dict__, "idx": model.idx.copy()})
    bad.idx[5] = model.n  # one column index past the end
    _refused(tmp_path, spec_file(bad), "column index out of range")
    bad = synth.Model(**{**model.__dict__, "ptr": model.ptr.copy()})
    bad.ptr[10] = bad.ptr[11] + 1  # decreasing offsets
    _refused(tmp_path, spec_file(bad), "CSR offsets")
    bad = synth.Model(**{**model.__dict__, "ptr": model.ptr.copy()})
    bad.ptr[0] = 1
    _refused(tmp_path, spec_file(bad), "CSR storage")


def test_writer_refuses_bad_models_and_paths(tmp_path):
    model = _lp()
    bad = synth.Model(**{**model.__dict__, "idx": model.idx.copy()})
    bad.idx[0] = -1
    with pytest.raises(engine.EngineError, match="column index out of range"):
        modelfile.save(bad, tmp_path / "bad.nkm")
    with pytest.raises(engine.EngineError, match="cannot create"):
        modelfile.save(model, tmp_path / "no" / "such" / "dir.nkm")
    assert not list(tmp_path.iterdir())


def test_command_line_convert_and_info(tmp_path, capsys):
    model = sparse_qp_model()
    src = tmp_path / "qp.json"
    src.write_text(json.dumps(serve._finite(serve.model_to_json(model))))
    assert modelfile._main(["convert", str(src), str(tmp_path / "qp.nkm")]) == 0
    _same(model, modelfile.load(tmp_path / "qp.nkm"))
    assert modelfile._main(["info", str(tmp_path / "qp.nkm")]) == 0
    assert "mapped and checked" in capsys.readouterr().out
    assert modelfile._main(["bogus"]) == 2


def _reference():
    from oracle import oracle
    try:
        return oracle.Reference()
    except FileNotFoundError:
        pytest.skip("reference library not built (make -C oracle ref)")


@pytest.mark.parametrize("make,sense", [(_lp, "min"), (sparse_qp_model, "min"), (_lp, "max")],
                         ids=["lp", "qp", "lp-max"])
def test_file_holds_what_the_reference_reads(tmp_path, make, sense):
    """The reference's read_model on the native JSON of a model builds exactly
    the arrays the model file converted from that JSON holds (the reference
    canonicalises to minimisation and sorts each CSR row)."""
    d = serve.model_to_json(make())
    d["sense"] = sense
    src = tmp_path / "model.json"
    src.write_text(json.dumps(serve._finite(d)))
    ref = _reference().read_model(src)
    assert modelfile._main(["convert", str(src), str(tmp_path / "model.nkm")]) == 0
    back = modelfile.load(tmp_path / "model.nkm")
    _same(ref, back)
    assert back.sense == (-1.0 if sense == "max" else 1.0)
