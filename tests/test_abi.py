"""CPU tests of the boundary: the C-ABI library loads without a GPU, exports
every entry point include/*.h declares, and the host-side mirror validates
its inputs.  No compute calls are made here."""
import ctypes as C
import glob
import os
import re

import pytest

from paratreet_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(pt_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    decl = declared_symbols()
    assert len(decl) >= 20
    missing = [n for n in sorted(decl) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_every_declared_symbol():
    assert declared_symbols() == set(L.SIGNATURES)


def test_abi_version_and_defaults_without_gpu():
    lib = L.load()
    assert lib.pt_abi_version() == 2
    cfg = L.PtConfig()
    assert lib.pt_config_default(C.byref(cfg)) == 0
    assert cfg.theta == 0.7 and cfg.bucket == 16 and cfg.dt_max == 1e-5
    assert lib.pt_config_default(None) == -1


def test_create_rejects_bad_config():
    lib = L.load()
    cfg = L.PtConfig()
    lib.pt_config_default(C.byref(cfg))
    h = C.c_void_p()
    cfg.bucket = 33
    assert lib.pt_create(C.byref(cfg), C.byref(h)) == -1
    cfg.bucket = 16
    cfg.theta = 0.0
    assert lib.pt_create(C.byref(cfg), C.byref(h)) == -1
    cfg.theta = 0.7
    cfg.traversal = 2  # neither PT_TRANSPOSED_DOWN nor PT_BASIC_DOWN
    assert lib.pt_create(C.byref(cfg), C.byref(h)) == -1
    cfg.traversal = L.PT_BASIC_DOWN
    # periodic: positive period, 0..8 replica shells, bounded cuts, no recorded lists
    cfg.periodic = 1
    assert (cfg.period, cfg.ewald_rcut, cfg.ewald_hcut) == (1.0, 2.6, 2.8)
    for field, bad in (("period", 0.0), ("n_replicas", 9), ("n_replicas", -1), ("record_lists", 1),
                       ("ewald_rcut", 0.0), ("ewald_rcut", 9.0), ("ewald_hcut", 17.0)):
        keep = getattr(cfg, field)
        setattr(cfg, field, bad)
        assert lib.pt_create(C.byref(cfg), C.byref(h)) == -1, field
        setattr(cfg, field, keep)


def test_null_handle_calls_return_errors():
    lib = L.load()
    assert lib.pt_compute_forces(None) == -1
    assert lib.pt_step(None, 1) == -1
    assert lib.pt_destroy(None) == 0
    assert lib.pt_sph_density(None, None, None, None, None) == -1
    assert lib.pt_sph_pressure(None, None, None, None, None, None, None) == -1
    assert lib.pt_sph_step(None, 1, None, None, None, None, None) == -1


def test_visitor_mirror():
    from paratreet_b200.gravity import GravityVisitor
    v = GravityVisitor((0, 0, 0), 0.7)
    assert v.CallSelfLeaf and v.TargetMustBeLeaf
    assert v.gravity_factor == (4.0 / 3.0) / (0.7 * 0.7)
    with pytest.raises(ValueError):
        GravityVisitor((0, 0, 0), 0.0)
