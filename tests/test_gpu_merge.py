"""Hit merging on the GPU (phx_merge_hits) against the numpy oracle, the reference's own SPM merge
run on the same device, the known-answer fixture and the simulated detector's hits."""
import numpy as np
import pytest

from oracle import merge as M
from oracle import oracle as O
from tests.test_merge import EC, SD, random_records

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng(cuda):
    from opticks_b200 import engine as E
    from opticks_b200 import scenes
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    e = E.Engine(fd.arrays(), phys, E.default_config(max_photon=200_000, num_sensor=scenes.NUM_PMT), device=0)
    yield e, lib
    e.close()


def same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("lite", [0, 1])
@pytest.mark.parametrize("mask,tw", [(0xFFFFFFFF, 1.0), (SD, 1.0), (SD, 0.5), (EC, 4.0), (SD, 1e9), (SD, 0.0), (0, 1.0)])
def test_merge_equals_oracle(eng, lite, mask, tw):
    e, _ = eng
    rng = np.random.default_rng(100 + lite)
    for n in (1, 31, 2048, 2049, 70_001):
        rec = random_records(n, lite, rng, num_id=60, tmax=40.0)
        assert same(e.merge_hits(rec, mask, tw), M.merge(rec, mask, tw)), (n, mask, tw)


@pytest.mark.parametrize("lite", [0, 1])
def test_merge_known_answer(eng, lite):
    e, _ = eng
    x = M.mock_merged(2000, 1.0, bool(lite))
    photons = M.unmerge(x)                                      # 2,001,000 records
    photons = photons[np.random.default_rng(42).permutation(len(photons))]
    assert same(e.merge_hits(photons, EC, 1.0), x)


@pytest.mark.skipif(not O.have_ref_spm(), reason="reference GPU build absent")
@pytest.mark.parametrize("lite", [0, 1])
@pytest.mark.parametrize("mask,tw", [(SD, 1.0), (SD, 0.37), (0xFFFFFFFF, 2.5), (SD, 0.0)])
def test_merge_equals_reference_spm(eng, lite, mask, tw):
    e, _ = eng
    rng = np.random.default_rng(7)
    rec = random_records(50_000, lite, rng, num_id=300, tmax=80.0, tq=0.01)
    ref = O.ref_merge_gpu(rec, mask, tw)
    got = e.merge_hits(rec, mask, tw)
    print(f"lite {lite} mask {mask:#x} window {tw}: {len(rec)} -> {len(got)} (reference {len(ref)})")
    assert same(got, ref)


def test_merge_detector_hits(eng):
    e, lib = eng
    from opticks_b200 import scenes
    gs = scenes.detector_gensteps(20, 5000, seed=3, lib=lib)
    r = e.simulate(gs, 0)
    ph = r["photon"]
    for tw in (1.0, 0.25, 10.0):
        got = e.merge_hits(ph, SD, tw)
        assert same(got, M.merge(ph, SD, tw))
        assert int((got.view(np.uint32)[:, 1, 3] >> 16).sum()) == r["num_hit"]   # every hit counted once
    # per-launch merges of two halves, then the final merge, equal one merge
    a = e.merge_hits(ph[: len(ph) // 2], SD, 1.0)
    b = e.merge_hits(ph[len(ph) // 2:], SD, 1.0)
    assert same(e.merge_hits(np.concatenate([a, b]), 0xFFFFFFFF, 1.0), e.merge_hits(ph, SD, 1.0))


def test_merge_device_api_and_errors(eng, cuda):
    torch = cuda
    e, _ = eng
    rng = np.random.default_rng(9)
    rec = random_records(30_000, 0, rng, num_id=50)
    d_in = torch.from_numpy(rec).cuda()
    d_out = torch.empty_like(d_in)
    n = e.merge_hits_device(d_in, d_out, SD, 1.0, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert same(d_out[:n].cpu().numpy(), M.merge(rec, SD, 1.0))
    with pytest.raises(ValueError):
        e.merge_hits_device(d_in, d_out[: n - 1], SD, 1.0)
    empty = torch.empty((0, 4), dtype=torch.float32, device="cuda")
    assert e.merge_hits_device(empty, empty, SD, 1.0) == 0
    with pytest.raises(RuntimeError):
        e.merge_hits(rec, SD, -1.0)


def test_merge_large(eng):
    e, _ = eng
    rng = np.random.default_rng(5)
    rec = random_records(4_000_000, 1, rng, num_id=17612, tmax=400.0, tq=0.001)
    got = e.merge_hits(rec, SD, 1.0)
    k = M.keys(got, 1.0)
    assert np.all(k[1:] > k[:-1])
    sel = (rec.view(np.uint32)[:, 3] & SD) != 0
    assert int((got.view(np.uint32)[:, 0] >> 16).sum()) == int((rec.view(np.uint32)[sel, 0] >> 16).sum())
    assert same(got, M.merge(rec, SD, 1.0))
