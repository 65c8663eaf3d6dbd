"""The C-ABI library loads and exports every entry point of include/dclaw_b200.h
(host-side calls only: no device work on the CPU runner)."""
import ctypes
import re
from pathlib import Path

from dclaw_b200 import _lib
from dclaw_b200.params import CParams, DClawParams

HEADER = Path(__file__).resolve().parents[1] / "include" / "dclaw_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(dclaw_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.SIGNATURES)


def test_host_side_helpers():
    lib = _lib.load()
    assert lib.dclaw_abi_version() == 2
    p = CParams()
    lib.dclaw_params_default(ctypes.byref(p))
    assert p.grav == 9.81 and p.limiter == 4 and p.order == 2
    assert lib.dclaw_params_check(ctypes.byref(p)) == 0
    mine = DClawParams().to_c()
    assert lib.dclaw_params_check(ctypes.byref(mine)) == 0
    bad = DClawParams(bed_normal=1).to_c()
    assert lib.dclaw_params_check(ctypes.byref(bad)) == 2
    bad = DClawParams(src2method=3).to_c()
    assert lib.dclaw_params_check(ctypes.byref(bad)) == 2
    # src2method 2 needs alphamethod 1, as the reference's setrun writer demands
    bad = DClawParams(src2method=2).to_c()
    assert lib.dclaw_params_check(ctypes.byref(bad)) == 1
    ok = DClawParams(src2method=2, alphamethod=1).to_c()
    assert lib.dclaw_params_check(ctypes.byref(ok)) == 0
    bad = DClawParams(order=3).to_c()
    assert lib.dclaw_params_check(ctypes.byref(bad)) == 1
    assert lib.dclaw_workspace_bytes(1, 10) == 0
    assert lib.dclaw_workspace_bytes(4096, 4096) > 0
    assert lib.dclaw_error_string(3) == b"NaN in the state"


def test_observation_record_argument_checks():
    """dclaw_obs_record refuses bad arguments before any device work."""
    lib = _lib.load()
    fake = ctypes.c_void_p(256)   # never dereferenced: every call below fails its checks
    null = ctypes.c_void_p(0)
    args = dict(clocks=fake, n=1, member=null, q=fake, sel=null, nsel=10, n_obs=4, step=1, out=fake, ostep=fake)

    def call(**kw):
        a = dict(args, **kw)
        return lib.dclaw_obs_record(a["clocks"], a["n"], a["member"], a["q"], a["sel"], a["nsel"], a["n_obs"],
                                    a["step"], a["out"], a["ostep"], null)

    for bad in (dict(clocks=null), dict(n=0), dict(q=null), dict(nsel=0), dict(n_obs=0), dict(out=null),
                dict(ostep=null), dict(n=3)):      # several clocks need a member map
        assert call(**bad) == 1, bad


def test_peak_argument_checks():
    lib = _lib.load()
    fake, null = ctypes.c_void_p(256), ctypes.c_void_p(0)
    assert lib.dclaw_peak_update(null, fake, fake, 10, 1, null) == 1
    assert lib.dclaw_peak_update(fake, fake, fake, 0, 1, null) == 1
    assert lib.dclaw_peak_adjoint(fake, null, 10, 1, fake, null) == 1
    assert lib.dclaw_peak_adjoint(fake, fake, 10, 1, null, null) == 1


def test_fortran_adapter_argument_checks():
    lib = _lib.load()
    fake, null = ctypes.c_void_p(256), ctypes.c_void_p(0)
    for fn in (lib.dclaw_fields_from_fortran, lib.dclaw_fields_to_fortran):
        for a, nfa, nf, mx, my, mbc, b in ((null, 7, 5, 8, 8, 2, fake), (fake, 7, 5, 8, 8, 2, null),
                                            (fake, 4, 5, 8, 8, 2, fake), (fake, 7, 0, 8, 8, 2, fake),
                                            (fake, 7, 5, 0, 8, 2, fake), (fake, 7, 5, 8, 8, -1, fake)):
            if fn is lib.dclaw_fields_to_fortran:
                assert fn(b, nf, nfa, mx, my, mbc, a, null) == 1
            else:
                assert fn(a, nfa, nf, mx, my, mbc, b, null) == 1


def test_ctypes_struct_matches_header_size():
    # dclaw_params: 8 doubles + 2 int32 + ... checked by field offsets of the ctypes image
    assert ctypes.sizeof(CParams) % 8 == 0
    assert CParams.bc_lower.offset % 4 == 0


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every ctypes image of a header struct has the C compiler's size and
    field offsets (a C probe compiled against include/dclaw_b200.h)."""
    import shutil
    import subprocess

    import pytest

    from dclaw_b200.params import CAdjBatch, CAdjMember, CBatch, CClock, CMember

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    images = {"dclaw_params": CParams, "dclaw_clock": CClock, "dclaw_member": CMember, "dclaw_batch": CBatch,
              "dclaw_adj_member": CAdjMember, "dclaw_adj_batch": CAdjBatch}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "dclaw_b200.h"', "int main(void) {"]
    for cname, img in images.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, *_ in img._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "probe"
    subprocess.run([cc, "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            cname, key, val = line.split()
            got[(cname, key)] = int(val)
    for cname, img in images.items():
        assert got[(cname, "size")] == ctypes.sizeof(img), cname
        for fname, *_ in img._fields_:
            assert got[(cname, fname)] == getattr(img, fname).offset, f"{cname}.{fname}"
