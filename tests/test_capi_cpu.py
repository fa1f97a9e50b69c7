"""Host-side checks of the C ABI library that need no GPU: it loads, exports
every declared entry point, and its host helpers (bit layout, .tns I/O, shard
planning, CLI argument handling) agree with the oracle / reference rules."""
import os
import re
import subprocess

import numpy as np
import pytest

import gsparc_b200 as gb
import oracle_bind as ob
from gsparc_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "gsparc_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gsparc_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = gb.lib()
    decl = _declared()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(L, name), name
    assert set(gb.EXPORTS) <= set(decl)


def test_ctypes_structs_match_the_header(tmp_path):
    """Sizes and field offsets of the Python binding's structs equal the C ones."""
    from gsparc_b200 import api
    structs = {"gsparc_coo": api._Coo, "gsparc_sink": api._Sink, "gsparc_stats": api.Stats,
               "gsparc_job": api._Job, "gsparc_digest": api.Digest,
               "gsparc_server_opts": api._ServerOpts, "gsparc_server_stats": api.ServeStats,
               "gsparc_tuning": api.Tuning}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "gsparc_b200.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "abi.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.split("\n") if l)
    for cname, py in structs.items():
        import ctypes
        assert int(out[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(out[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"


def test_version_and_status_strings():
    assert "sm_100a" in gb.version()
    assert gb.lib().gsparc_status_string(2) == b"out of memory"


@pytest.mark.parametrize("dims,cm", [([2482, 2862, 14036, 17], [2, 3]), ([13, 40, 17], [2, 1]),
                                     ([1000, 1000, 1000], [2]), ([7, 1, 9, 2], [3, 0]),
                                     ([2**40, 2**20, 3], [1])])
def test_layout_matches_oracle(dims, cm):
    bits, shift, isc, ncb, nfb = gb.layout(dims, cm)
    oshift, oisc, oncb, onfb = ob.layout(dims, cm)
    assert (ncb, nfb) == (oncb, onfb)
    assert list(shift) == list(oshift) and list(isc) == list(oisc)
    assert list(bits) == [ob.mode_bits(d) for d in dims]


def test_layout_rejects_bad_modes():
    with pytest.raises(gb.GsparcError):
        gb.layout([10, 10], [2])
    with pytest.raises(gb.GsparcError):
        gb.layout([10, 10, 10], [1, 1])


@pytest.mark.parametrize("seed", [0, 1])
def test_read_tns_matches_oracle_parser(tmp_path, seed):
    t = synth.make_tensor([50, 7, 300], 3000, ["uniform", ("zipf", 1.3), "uniform"], "normal", seed)
    p = str(tmp_path / "a.tns")
    synth.write_tns(p, t)
    a = gb.read_tns(p, nthreads=4)
    b = ob.read_tns(p)
    assert a.dims == b.dims == t.dims
    assert np.array_equal(a.idx, b.idx) and np.array_equal(a.idx, t.idx)
    assert np.array_equal(a.val, b.val) and np.array_equal(a.val, t.val)


def test_read_tns_tolerates_blank_lines_tabs_crlf(tmp_path):
    p = tmp_path / "b.tns"
    p.write_bytes(b"1\t2 3 0.5\r\n\n  4 5 6\t-1.25e-3\r\n2 2 2 7\n\n")
    a = gb.read_tns(str(p), nthreads=3)
    assert a.dims == [4, 5, 6]
    assert a.idx.tolist() == [[0, 3, 1], [1, 4, 1], [2, 5, 1]]
    assert np.allclose(a.val, [0.5, -1.25e-3, 7.0])


@pytest.mark.parametrize("content", [b"1 2 3\n0 1 1 2.0\n", b"1 2 3 1.0\n1 2\n", b"",
                                     b"1 x 3 1.0\n"])
def test_read_tns_reports_malformed_input(tmp_path, content):
    p = tmp_path / "bad.tns"
    p.write_bytes(content)
    with pytest.raises(gb.GsparcError) as e:
        gb.read_tns(str(p))
    assert e.value.status == 1


def test_read_tns_missing_file():
    with pytest.raises(gb.GsparcError) as e:
        gb.read_tns("/nonexistent/x.tns")
    assert e.value.status == 4


def test_write_tns_round_trip(tmp_path):
    t = synth.make_tensor([9, 99, 999], 500, ["uniform"] * 3, "u11", 5)
    p = str(tmp_path / "w.tns")
    gb.write_tns(p, t.idx, t.val)
    a = gb.read_tns(p)
    assert np.array_equal(a.idx, t.idx) and np.array_equal(a.val, t.val)


def test_plan_shards_balances_product_mass():
    rng = np.random.default_rng(0)
    rp = (rng.pareto(1.2, 100000) * 100).astype(np.uint64)
    for n in (1, 2, 4, 8):
        b = gb.plan_shards(rp, n)
        assert b[0] == 0 and b[-1] == rp.shape[0] and np.all(np.diff(b.astype(np.int64)) >= 0)
        mass = [int(rp[b[i]:b[i + 1]].sum()) for i in range(n)]
        assert sum(mass) == int(rp.sum())
        assert max(mass) <= int(rp.sum()) / n + int(rp.max())
    assert list(gb.plan_shards(np.zeros(0, np.uint64), 3)) == [0, 0, 0, 0]


def test_context_without_gpu_returns_status_not_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(gb.GsparcError) as e:
        gb.Context(0)
    assert e.value.status in (1, 3)


def test_cli_rejects_unsupported_and_bad_arguments(tmp_path):
    cli = gb.CLI_PATH
    assert os.path.exists(cli)
    r = subprocess.run([cli, "-X", "/none/qa", "-Y", "/none/qb", "-c", "1", "-x", "0", "-y", "0", "-q"],
                       capture_output=True, text=True)
    assert r.returncode == 1 and "indices.txt" in r.stderr
    # chained multi-SpTC runs on one GPU and needs -a/-z consistent with Y
    d = tmp_path
    synth.write_tns(str(d / "a.tns"), synth.make_tensor([5, 6, 7], 20, ["uniform"] * 3, "u01", 1))
    r = subprocess.run([cli, "-X", str(d / "a.tns"), "-Y", str(d / "a.tns"), "-c", "1", "-x", "2", "-y", "2",
                        "-m", "1", "-a", "1", "-z", "0", "-g", "2"], capture_output=True, text=True)
    assert r.returncode == 1 and "one GPU" in r.stderr
    assert "multi_sptc: 1" in r.stderr and "# contract modes of Z (second SpTC): 1, contract modes: 0 \n" in r.stderr
    r = subprocess.run([cli, "-X", str(d / "a.tns"), "-Y", str(d / "a.tns"), "-c", "1", "-x", "2", "-y", "2",
                        "-m", "1", "-a", "3", "-z", "0", "1", "2"], capture_output=True, text=True)
    assert r.returncode == 1 and "-a N" in r.stderr
    r = subprocess.run([cli, "-X", "a"], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
    r = subprocess.run([cli, "-X", "/none/a.tns", "-Y", "/none/b.tns", "-c", "2", "-x", "0", "1",
                        "-y", "1", "0", "-d", "-1"], capture_output=True, text=True)
    assert r.returncode == 1
    # the reference's parse-time report lines (src/gsparc/cmdline_opts.cpp:92-171)
    assert "tensor X: /none/a.tns" in r.stderr and "tensor Y: /none/b.tns" in r.stderr
    assert "# contract modes of X: 2, contract modes: 0 1 \n" in r.stderr
    assert "# contract modes of Y: 2, contract modes: 1 0 \n" in r.stderr
    assert "dense_accumulator: -1" in r.stderr


@pytest.mark.parametrize("seed", [0, 1])
def test_read_quantum_matches_oracle_parser(tmp_path, seed):
    t = synth.make_tensor([30, 7, 120, 9], 400, ["uniform", ("zipf", 1.2), "uniform", "uniform"], "normal", seed)
    d = str(tmp_path / "q")
    synth.write_quantum(d, t)
    a = gb.read_quantum(d)
    b = ob.read_quantum(d)
    assert a.dims == b.dims == t.dims
    assert np.array_equal(a.idx, b.idx) and np.array_equal(a.idx, t.idx)
    assert np.array_equal(a.val, b.val) and np.array_equal(a.val, t.val)
    # the same tensor through .tns reads identically
    p = str(tmp_path / "t.tns")
    synth.write_tns(p, t)
    c = gb.read_tns(p)
    assert c.dims == a.dims and np.array_equal(c.idx, a.idx) and np.array_equal(c.val, a.val)


def test_read_quantum_number_formats_and_blank_lines(tmp_path):
    d = tmp_path / "q"
    d.mkdir()
    (d / "indices.txt").write_text("1 3.0\t2\n\n4 4 1\r\n")
    (d / "values.txt").write_text("1.5e0\n-2.25\n\n3E-1\n")
    a = gb.read_quantum(str(d))
    b = ob.read_quantum(str(d))
    assert a.dims == b.dims == [3, 4]
    assert a.idx.tolist() == b.idx.tolist() == [[0, 2, 1], [3, 3, 0]]
    assert a.val.tolist() == b.val.tolist() == [1.5, -2.25, np.float32(0.3)]


@pytest.mark.parametrize("idx,vals", [("1 2\n1\n", "1 2\n"),        # lines of different lengths
                                      ("1 0\n1 1\n", "1 2\n"),      # index 0 (indices are 1-based)
                                      ("1 2.5\n1 1\n", "1 2\n"),    # non-integral index
                                      ("1 2\n1 1\n", "1\n"),         # fewer values than nonzeros
                                      ("", "")])                         # no modes
def test_read_quantum_reports_malformed_input(tmp_path, idx, vals):
    d = tmp_path / "q"
    d.mkdir()
    (d / "indices.txt").write_text(idx)
    (d / "values.txt").write_text(vals)
    with pytest.raises(gb.GsparcError) as e:
        gb.read_quantum(str(d))
    assert e.value.status == 4
    with pytest.raises(ValueError):
        ob.read_quantum(str(d))


def test_read_quantum_missing_directory():
    with pytest.raises(gb.GsparcError) as e:
        gb.read_quantum("/none/such/dir")
    assert e.value.status == 4


def test_served_stream_generator():
    inst, arrive = synth.served_stream(count=40, seed=2, max_nnz=5_000, min_nnz=500)
    assert len(inst) == 40 and np.all(np.diff(arrive) > 0)
    orders = set()
    for X, Y, cx, cy in inst:
        orders |= {X.order, Y.order}
        assert 1 <= len(cx) == len(cy) <= 2
        assert [X.dims[m] for m in cx] == [Y.dims[m] for m in cy]
        fx = [d for m, d in enumerate(X.dims) if m not in cx]
        fy = [d for m, d in enumerate(Y.dims) if m not in cy]
        assert sum(synth._bits(d) for d in fx + fy) <= 64
        assert 1 <= X.nnz <= 5_000 and 1 <= Y.nnz <= 5_000
    assert orders <= {3, 4, 5} and len(orders) >= 2
