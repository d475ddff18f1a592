"""Delimited integer baskets parsed on the device (cpm_parse_int_text) against
the CPU reader, which restates the reference's csv.reader path.

The reference reads such files with cuDF when it can (_gpu_io.py:34-54) and
with csv.reader otherwise; both give the same baskets for unquoted integer
layouts.  Here the device parse must give, basket for basket, what the CPU
reader gives -- blank lines, spaces around separators, CRLF endings, a last
line without a newline, tabs or commas -- and anything outside the layout
(quotes, leading zeros, letters, empty tokens) must be left to the CPU reader.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _baskets_of(miner):
    off, ids = miner._csr
    o = off.astype(np.int64)
    return [tuple(str(v) for v in ids[o[k]:o[k + 1]].tolist()) for k in range(o.size - 1) if o[k + 1] > o[k]]


def _write_random(path, rng, sep, crlf=False, spaces=False, trailing=True):
    lines = []
    for _ in range(3000):
        n = rng.poisson(4)
        items = rng.zipf(1.3, n) % 5000
        if rng.random() < 0.05:
            lines.append("  " if spaces else "")
            continue
        glue = (" " + sep + " ") if spaces and rng.random() < 0.5 else sep
        lines.append(glue.join(str(int(x)) for x in items))
    text = ("\r\n" if crlf else "\n").join(lines) + (("\r\n" if crlf else "\n") if trailing else "")
    path.write_text(text, encoding="utf-8")


@pytest.mark.parametrize("sep,crlf,spaces,trailing", [(",", False, False, True), ("\t", True, True, False),
                                                     (",", True, True, True), (" ", False, False, False)])
def test_device_text_matches_cpu_reader(tmp_path, sep, crlf, spaces, trailing):
    import cupami_b200

    rng = np.random.default_rng(ord(sep) + 2 * crlf + 4 * spaces + 8 * trailing)
    path = tmp_path / "b.csv"
    _write_random(path, rng, sep, crlf, spaces, trailing)
    explicit = sep if sep == " " else None
    dev = cupami_b200.cuEclat(path, 0.01, explicit)
    cpu = cupami_b200.cuEclat(path, 0.01, explicit, use_gpu_io=False)
    assert dev.getInputBackend()["backend"] == "cuda-text"
    want = [tuple(dict.fromkeys(b)) for b in cpu._Database]
    got = _baskets_of(dev)
    assert [tuple(dict.fromkeys(b)) for b in got] == want
    assert dev._transactionCount == cpu._transactionCount and dev._minSup == cpu._minSup
    dev.mine()
    cpu.mine()
    assert dev.getPatterns() == cpu.getPatterns()


@pytest.mark.parametrize("text", ['1,2\n"3",4\n', "1,07\n", "1,a\n", "1,,2\n", "1,2,\n", "4294967296\n",
                                  "\ufeff1,2\n"])
def test_other_layouts_go_to_the_cpu_reader(tmp_path, text):
    import cupami_b200
    from cupami_b200 import _native

    path = tmp_path / "o.csv"
    path.write_text(text, encoding="utf-8")
    m = cupami_b200.cuApriori(path, 1)
    assert m.getInputBackend()["backend"] == "cpu"
    assert m._csr is None
    with pytest.raises(_native.NativeError):
        _native.parse_int_text(_native.context(0), text.encode("utf-8"), ",")
    with pytest.raises(RuntimeError):
        cupami_b200.cuApriori(path, 1, use_gpu_io=True)


def test_empty_and_blank_text():
    from cupami_b200 import _native

    ctx = _native.context(0)
    off, ids = _native.parse_int_text(ctx, b"", ",")
    assert off.tolist() == [0] and ids.size == 0
    off, ids = _native.parse_int_text(ctx, b"\n  \n\t\n5\n", ",")
    assert off.tolist() == [0, 0, 0, 0, 1] and ids.tolist() == [5]
    off, ids = _native.parse_int_text(ctx, b"0, 4294967295 ,12", ",")
    assert off.tolist() == [0, 3] and ids.tolist() == [0, 4294967295, 12]
