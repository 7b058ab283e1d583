"""The C ABI library: it loads without a GPU, exports every symbol include/phox.h declares,
and fails loudly (an error, never a CPU fallback) when no device is present."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "phox.h")
LIB = os.path.join(ROOT, "opticks_b200", "libphox.so")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(phx_[a-z0-9_]+)\s*\(", txt)))


def test_library_builds_and_exports_every_declared_symbol():
    from opticks_b200 import build
    build.build()
    assert os.path.exists(LIB)
    syms = declared_symbols()
    assert len(syms) >= 12
    nm = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (phx_\w+)", nm))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    lib = C.CDLL(LIB)
    for s in syms:
        assert getattr(lib, s) is not None


def test_ctypes_signatures_cover_header():
    from opticks_b200 import _lib
    assert set(_lib.SIGNATURES) == set(declared_symbols())


def test_config_defaults_match_reference_eventconfig():
    from opticks_b200 import engine as E
    c = E.default_config()
    assert c.max_bounce == 31 and c.skipahead_event_offset == 100000
    assert abs(c.propagate_epsilon - 0.05) < 1e-7 and abs(c.propagate_epsilon0 - 0.05) < 1e-7
    assert c.hit_mask == E.FLAG["SD"]
    assert c.epsilon0_mask == E.mask_from_labels("TO,CK,SI,SC,RE")
    assert c.max_time > 1e26


def test_count_photons():
    from opticks_b200 import _lib, scenes
    gs = np.concatenate([scenes.torch_genstep(7)[None], scenes.torch_genstep(11)[None]])
    assert _lib.lib().phx_count_photons(gs.ctypes.data_as(C.c_void_p), 2) == 18


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from opticks_b200 import engine as E, scenes
    fd, lib, icdf, gs = scenes.sphere_in_box(10)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        E.Engine(fd.arrays(), lib.arrays())
