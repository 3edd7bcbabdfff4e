"""The C-ABI library loads without a GPU and exports every entry point include/*.h declares."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(lbg_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    assert "lbg_commit" in declared() and "lbg_fold" in declared()


def test_library_exports_every_declared_symbol(native):
    lib = native.lib()
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert missing == []


def test_bindings_cover_every_declared_symbol(native):
    assert sorted(set(declared()) - set(native.SIGNATURES)) == []


def test_library_exports_nothing_else():
    import subprocess

    from labinius_b200 import _native

    out = subprocess.run(["nm", "-D", "--defined-only", _native.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert {n for n in exported if n.startswith("lbg_")} == set(declared())


def test_params_check_mirrors_param_error(native):
    """crates/pcs/tests/api.rs:47-126"""
    import ctypes

    def P(wl, cl, moduli, opening=0, bits=0):
        p = native.lbg_params()
        p.witness_log_len, p.column_log_len, p.n_moduli = wl, cl, len(moduli)
        for i, q in enumerate(moduli):
            p.moduli[i] = q
        p.opening, p.dropped_bits = opening, bits
        return native.lib().lbg_params_check(ctypes.byref(p))

    assert P(18, 7, [3889, 9721]) == 0
    assert P(18, 19, [3889]) == native.LBG_ERR_PARAMS
    assert P(18, 0, [3889]) == native.LBG_ERR_PARAMS
    assert P(10, 4, [3889]) == native.LBG_ERR_PARAMS
    assert P(18, 7, [3889, 3889]) == native.LBG_ERR_PARAMS
    assert P(18, 7, [3889, 9721, 9721]) == native.LBG_ERR_PARAMS
    assert P(18, 7, [3889, 1234]) == native.LBG_ERR_PARAMS
    # Opening::Recursive validates like the other openings (crates/pcs/src/scheme/params.rs:171-203)
    assert P(18, 8, [3889, 2917, 4861], opening=2) == 0
    assert P(18, 19, [3889], opening=2) == native.LBG_ERR_PARAMS
    assert P(18, 7, [3889], opening=3) == native.LBG_ERR_PARAMS
    assert P(18, 7, [3889, 2917, 4861], opening=1, bits=9) == 0


def test_python_params_mirror():
    from labinius_b200 import SUITES, Modulus, Opening, ParamError, Params

    b = Params.basic()
    assert (b.witness_log_len, b.base, b.extra_moduli, b.columns()) == (18, Modulus.Q3889_FS_S, [Modulus.Q9721_FS_S], 128)
    assert b.primes() == [3889, 9721]
    l = Params.sized(SUITES[2], Opening.clear())
    assert (l.witness_len(), l.columns(), l.primes()) == (1 << 22, 512, [3889, 2917, 4861])
    xl = Params.sized(SUITES[3], Opening.clear())
    assert xl.primes() == [3889, 2917, 9721]
    for bad in [(18, 19, []), (18, 0, []), (10, 4, [])]:
        with pytest.raises(ParamError):
            Params.new(*bad)
    with pytest.raises(ParamError):
        Params.new(18, 7, [Modulus.Q3889_FS_S])
    with pytest.raises(ParamError):
        Params.new(18, 7, [Modulus.Q9721_FS_S, Modulus.Q9721_FS_S])
