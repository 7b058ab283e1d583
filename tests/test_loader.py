"""Reference on-disk layout: CSGFoundry/*.npy + SSim/stree/standard/{bnd,optical,icdf}.npy with the
bnd_meta.txt domain sidecar — write, read back bit for bit, reject malformed directories, and run
the CPU oracle on the loaded arrays."""
import os

import numpy as np
import pytest

from opticks_b200 import loader, scenes


@pytest.fixture(scope="module")
def det():
    fd, lib, icdf = scenes.detector(num_pmt=300)
    phys = lib.arrays()
    phys["icdf"] = icdf
    return fd, lib, phys


def test_round_trip(det, tmp_path):
    fd, lib, phys = det
    geom = fd.arrays()
    loader.save_geom(str(tmp_path), geom, phys, meshname=["global", "pmt"], bnd_names=["a", "b", "c", "d"])
    fold = os.path.join(tmp_path, "CSGFoundry")
    for k in ("solid", "prim", "node", "tran", "itra", "inst"):
        assert os.path.exists(os.path.join(fold, f"{k}.npy"))
    std = os.path.join(fold, "SSim", "stree", "standard")
    assert open(os.path.join(std, "bnd_meta.txt")).read().splitlines()[:3] == ["domain_low:60.0", "domain_high:820.0", "domain_step:1.0"]
    g2, p2 = loader.load_geom(str(tmp_path))
    for k in ("solid", "prim", "node", "tran", "itra", "inst"):
        assert np.array_equal(np.asarray(geom[k]).view(np.uint32), g2[k].view(np.uint32)), k
    assert g2["solid"].dtype == np.int32 and g2["node"].dtype == np.float32
    assert g2["meshname"] == ["global", "pmt"]
    assert np.array_equal(phys["bnd"], p2["bnd"]) and np.array_equal(phys["optical"], p2["optical"])
    assert np.array_equal(phys["icdf"], p2["icdf"])
    assert (p2["wl_low"], p2["wl_step"], p2["hd_factor"]) == (60.0, 1.0, 20)
    assert p2["bnd_names"] == ["a", "b", "c", "d"]


def test_rejects_malformed(det, tmp_path):
    fd, lib, phys = det
    loader.save_geom(str(tmp_path), fd.arrays(), phys)
    fold = os.path.join(tmp_path, "CSGFoundry")
    std = os.path.join(fold, "SSim", "stree", "standard")
    np.save(os.path.join(fold, "node.npy"), np.zeros((5, 3, 4), np.float32))
    with pytest.raises(ValueError):
        loader.load_foundry(fold)
    os.remove(os.path.join(fold, "node.npy"))
    with pytest.raises(FileNotFoundError):
        loader.load_foundry(fold)
    os.remove(os.path.join(std, "bnd_meta.txt"))
    with pytest.raises(ValueError):
        loader.load_standard(std)
    with pytest.raises(FileNotFoundError):
        loader.load_foundry(os.path.join(tmp_path, "nowhere"))


def test_oracle_on_loaded_arrays(det, tmp_path):
    from oracle import oracle as O
    fd, lib, phys = det
    loader.save_geom(str(tmp_path), fd.arrays(), phys)
    g2, p2 = loader.load_geom(str(tmp_path))
    gs = scenes.detector_gensteps(2, 100, seed=3, lib=lib)
    u = np.random.default_rng(1).random((200, 256), dtype=np.float32)
    a = O.Scene(fd.arrays(), phys).simulate(gs, u, 0)
    b = O.Scene({k: v for k, v in g2.items() if isinstance(v, np.ndarray)}, p2).simulate(gs, u, 0)
    assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32)) and np.array_equal(a[1], b[1])
