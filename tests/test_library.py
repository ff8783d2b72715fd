"""CPU checks of the product library: it loads, exports every entry point
include/mdg.h declares, builds spline tables bitwise equal to the oracle's,
and refuses to compute without a device."""
import ctypes
import os
import re

import numpy as np
import pytest

import mdtk_b200 as M
from oracle import ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if not name.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", name)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        syms |= set(re.findall(r"\b(mdg_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_library_loads_and_exports_all_declared_symbols():
    L = M.lib()
    syms = declared_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


@pytest.mark.skipif(not ref.available(), reason="oracle not built")
def test_rebo_tables_bitwise_equal_to_oracle():
    a = M.debug_rebo_tables()
    b = ref.tables(0)
    assert a.shape == b.shape
    assert np.array_equal(a, b)


@pytest.mark.skipif(not ref.available(), reason="oracle not built")
@pytest.mark.parametrize("bset", [1, 2])
def test_brenner_tables_bitwise_equal_to_oracle(bset):
    a = M.debug_brenner_tables(bset)
    b = ref.tables(1, bset)
    assert a.shape == b.shape
    assert np.array_equal(a, b)


def test_default_params():
    p = M.Params()
    M.lib().mdg_default_params(ctypes.byref(p))
    assert p.potentials == M.POT_REBO and p.precision == M.PREC_FP64 and p.units == M.UNITS_AEVFS


def test_create_rejects_lj_without_rebo():
    with pytest.raises(M.MdgError) as e:
        M.Context(potentials=M.POT_AIREBO_LJ)
    assert e.value.code == -1


def test_create_rejects_mixed_brenner():
    # checked before any device work, so it runs without a GPU
    with pytest.raises(M.MdgError) as e:
        M.Context(potentials=M.POT_BRENNER, precision=M.PREC_FP32_MIXED)
    assert e.value.code == -1


@pytest.mark.parametrize("kind,nfam", [(0, 3), (1, 2), (2, 4)])
def test_fp32_spline_tables_match_fp64(kind, nfam):
    # The FP32 tables re-expand every cell about its corner; over the domain
    # they agree with the FP64 (reference-order) evaluation to a few float ulps
    # of each family's scale.
    rng = np.random.default_rng(kind)
    n = 4000
    if kind == 0:
        a = rng.uniform(-1, 1, (n, 1))
    elif kind == 1:
        a = rng.uniform(0, 4, (n, 2))
    else:
        a = np.column_stack([rng.uniform(0, 4, n), rng.uniform(0, 4, n), rng.uniform(1, 12, n)])
    for fam in range(nfam):
        d = M.debug_spline(M.PREC_FP64, kind, fam, a)
        f = M.debug_spline(M.PREC_FP32_MIXED, kind, fam, a)
        scale = np.maximum(np.abs(d).max(axis=0), 1e-30)
        assert np.all(np.abs(f - d).max(axis=0) <= 5e-6 * scale), (kind, fam)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a device is present")
def test_no_device_fails_loudly():
    with pytest.raises(M.MdgError) as e:
        M.Context(potentials=M.POT_REBO)
    assert e.value.code == -2


def test_timeline_names_every_kernel_entry():
    # the timeline build keys its stamps by the source line of pdl_enter();
    # every such line in mdg_api.cu maps to the kernel that opens it
    from mdtk_b200 import timeline
    names = timeline.kernel_names()
    assert len(names) >= 30
    assert "?" not in names.values()
    for k in ("k_step_start", "k_lj_near", "k_lj_filter", "k_lj_pairs", "k_lj_special_pair", "k_gather_vv"):
        assert k in names.values(), k
