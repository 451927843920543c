"""The C ABI library loads and exports what include/gsofa.h declares; the
host-only entry points behave (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import gsofa_b200
from tests.common import bundled

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(gsofa_\w+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(gsofa_b200.LIB_PATH)
    declared = _declared()
    assert declared, "no declarations found"
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    assert set(gsofa_b200.exported_symbols()) <= declared


def test_abi_version_and_status_strings():
    L = gsofa_b200.lib()
    assert L.gsofa_abi_version() == 1
    for s in range(8):
        assert L.gsofa_status_str(s)
    p = gsofa_b200.Params.default()
    assert p.want_pattern == 1 and p.part_count == 1 and p.reuse == -1


def test_params_layout_matches_header(tmp_path):
    """The ctypes mirrors have the C structs' sizes and field offsets, as the
    C compiler lays them out from include/gsofa.h."""
    mirrors = {"gsofa_params": gsofa_b200.Params, "gsofa_result": gsofa_b200._CResult,
               "gsofa_supernodal": gsofa_b200._CSupernodal, "gsofa_server_config": gsofa_b200.ServerConfig}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "gsofa.h"', "int main(void) {"]
    for cname, mirror in mirrors.items():
        lines.append(f'printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f, _ in mirror._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)],
                   check=True)
    got = {}
    for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, field, val = line.split()
        got[(cname, field)] = int(val)
    for cname, mirror in mirrors.items():
        assert ctypes.sizeof(mirror) == got[(cname, "sizeof")], cname
        for f, _ in mirror._fields_:
            assert getattr(mirror, f).offset == got[(cname, f)], f"{cname}.{f}"


def test_read_text_matches_fixture(tmp_path):
    g = bundled()
    (tmp_path / "b.dat").write_text(" ".join(map(str, g.beg.tolist())) + "\n")
    (tmp_path / "e.dat").write_text(" ".join(map(str, g.end.tolist())) + "\n")
    (tmp_path / "c.dat").write_text(f"{g.nnz}\n{g.n}\n" + "\n".join(map(str, g.adj.tolist())) + "\n")
    r = gsofa_b200.read_text(str(tmp_path / "b.dat"), str(tmp_path / "e.dat"), str(tmp_path / "c.dat"))
    assert r.n == g.n and np.array_equal(r.beg, g.beg) and np.array_equal(r.end, g.end)
    assert np.array_equal(r.adj, g.adj)


def test_binary_files_round_trip_and_mix_with_text(tmp_path):
    g = bundled()
    p = {k: str(tmp_path / f"{k}.bin") for k in "bec"}
    gsofa_b200.write_binary(g, p["b"], p["e"], p["c"])
    assert open(p["c"], "rb").read(8) == b"GSOFAB01"
    r = gsofa_b200.read_text(p["b"], p["e"], p["c"])
    assert r.n == g.n and np.array_equal(r.beg, g.beg) and np.array_equal(r.end, g.end)
    assert np.array_equal(r.adj, g.adj)
    # a text colend beside binary colbeg and csr
    (tmp_path / "e.dat").write_text(" ".join(map(str, g.end.tolist())) + "\n")
    r = gsofa_b200.read_text(p["b"], str(tmp_path / "e.dat"), p["c"])
    assert np.array_equal(r.end, g.end) and np.array_equal(r.adj, g.adj)
    # a binary colbeg whose count disagrees with the csr header is an I/O error
    small = gsofa_b200.matgen.grid2d(4)
    gsofa_b200.write_binary(small, str(tmp_path / "sb.bin"), str(tmp_path / "se.bin"), str(tmp_path / "sc.bin"))
    with pytest.raises(gsofa_b200.GsofaError) as e:
        gsofa_b200.read_text(str(tmp_path / "sb.bin"), p["e"], p["c"])
    assert e.value.status == 6
    # truncated binary ids
    data = open(p["c"], "rb").read()
    open(str(tmp_path / "cut.bin"), "wb").write(data[: len(data) - 8])
    with pytest.raises(gsofa_b200.GsofaError):
        gsofa_b200.read_text(p["b"], p["e"], str(tmp_path / "cut.bin"))


def test_read_text_errors(tmp_path):
    with pytest.raises(gsofa_b200.GsofaError) as e:
        gsofa_b200.read_text(str(tmp_path / "nope"), str(tmp_path / "nope"), str(tmp_path / "nope"))
    assert e.value.status == 6
    (tmp_path / "c.dat").write_text("10\n5\n1 2 3\n")  # truncated
    (tmp_path / "b.dat").write_text("0 0 0 0 0")
    with pytest.raises(gsofa_b200.GsofaError):
        gsofa_b200.read_text(str(tmp_path / "b.dat"), str(tmp_path / "b.dat"), str(tmp_path / "c.dat"))


def test_bad_argv_is_a_status_not_an_exit():
    with pytest.raises(gsofa_b200.GsofaError) as e:
        gsofa_b200.symbfact_min_id(["gsofa", "a", "b"])
    assert e.value.status == 1


def test_cli_usage():
    cli = os.path.join(ROOT, "gsofa_b200", "gsofa")
    assert os.path.exists(cli)
    r = subprocess.run([cli], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr and "--to-binary" in r.stderr


def test_cli_converts_text_to_binary(tmp_path):
    g = bundled()
    (tmp_path / "b.dat").write_text(" ".join(map(str, g.beg.tolist())))
    (tmp_path / "e.dat").write_text(" ".join(map(str, g.end.tolist())))
    (tmp_path / "c.dat").write_text(f"{g.nnz} {g.n}\n" + " ".join(map(str, g.adj.tolist())))
    cli = os.path.join(ROOT, "gsofa_b200", "gsofa")
    pre = str(tmp_path / "m")
    r = subprocess.run([cli, "--to-binary", str(tmp_path / "b.dat"), str(tmp_path / "e.dat"),
                        str(tmp_path / "c.dat"), pre], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    back = gsofa_b200.read_text(pre + ".colbeg.bin", pre + ".colend.bin", pre + ".csr.bin")
    assert back.n == g.n and np.array_equal(back.adj, g.adj) and np.array_equal(back.beg, g.beg)
    r = subprocess.run([cli, "--to-binary", str(tmp_path / "nope"), str(tmp_path / "e.dat"),
                        str(tmp_path / "c.dat"), pre], capture_output=True, text=True)
    assert r.returncode == 1
