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
    assert open(os.path.join(std, "bnd_meta.txt")).read().splitlines()[:3] == ["domain_low:60", "domain_high:820", "domain_step:1"]
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


NPFOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "npfold")


def test_reads_files_the_reference_writer_made():
    """tests/golden/npfold was written by the reference's own sysrap/NP.hh in the shapes, dtypes and
    metadata of CSGFoundry::save_ and sstandard (plan (n,1,4), bnd float64 with its domain metadata,
    optical int32 (num_bnd,4,4), icdf float64): the loader gives back the arrays it was made from"""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_npfold import fixture_scene
    geom, phys, names = fixture_scene()
    g2, p2 = loader.load_geom(NPFOLD)
    for k in ("solid", "prim", "node", "itra", "inst", "plan"):
        assert g2[k].shape == np.asarray(geom[k]).shape, k
        np.testing.assert_array_equal(g2[k].view(np.uint32), np.ascontiguousarray(geom[k]).view(np.uint32), err_msg=k)
    assert p2["bnd"].dtype == np.float32
    np.testing.assert_array_equal(p2["bnd"], phys["bnd"])
    np.testing.assert_array_equal(p2["optical"], phys["optical"])
    np.testing.assert_array_equal(p2["icdf"], phys["icdf"])
    assert p2["wl_low"] == 60.0 and p2["wl_step"] == 1.0
    assert p2["bnd_names"] == names
    assert g2["meshname"] == [f"zoo_{k}" for k in range(len(geom["prim"]))]


def test_writer_matches_the_reference_layout(tmp_path):
    """save_geom writes what the reference's writer wrote: same shapes, dtypes and metadata keys"""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_npfold import fixture_scene
    geom, phys, names = fixture_scene()
    loader.save_geom(str(tmp_path), geom, phys, bnd_names=names)
    mine = os.path.join(tmp_path, "CSGFoundry")
    ref = os.path.join(NPFOLD, "CSGFoundry")
    for rel in ("solid.npy", "prim.npy", "node.npy", "itra.npy", "inst.npy", "plan.npy",
                "SSim/stree/standard/bnd.npy", "SSim/stree/standard/optical.npy", "SSim/stree/standard/icdf.npy"):
        a, b = np.load(os.path.join(mine, rel)), np.load(os.path.join(ref, rel))
        assert a.shape == b.shape and a.dtype == b.dtype, rel
        np.testing.assert_array_equal(a, b, err_msg=rel)
    assert loader.read_meta(os.path.join(mine, "SSim/stree/standard/bnd.npy")) == \
        loader.read_meta(os.path.join(ref, "SSim/stree/standard/bnd.npy"))
