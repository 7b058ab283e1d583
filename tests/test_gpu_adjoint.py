"""Score-function adjoint of the expected hits per sensor (phx_adjoint_device, torch autograd):
its forward equals the plain engine on the re-tabulated tables, its score sums equal the FP64 CPU
estimator on the same photons, and its gradient agrees with central finite differences under
common random numbers within the statistical error."""
import numpy as np
import pytest

from oracle import oracle as O
from opticks_b200 import adjoint as ADJ
from opticks_b200 import scenes

pytestmark = pytest.mark.gpu
WL = (300.0, 620.0)


@pytest.fixture(scope="module")
def det(cuda):
    torch = cuda
    from opticks_b200 import engine as E
    fd, lib, icdf = scenes.detector()
    phys = lib.arrays()
    phys["icdf"] = icdf
    mat_line = lib.material_line("LS")
    theta = ADJ.nominal_theta(phys, mat_line, *WL)
    eng = E.Engine(fd.arrays(), phys, E.default_config(max_photon=200_000, num_sensor=scenes.NUM_PMT))
    yield dict(torch=torch, E=E, fd=fd, lib=lib, phys=phys, mat_line=mat_line, theta=theta, eng=eng)
    eng.close()


def _adj(d, gs, theta, event=0, pathwise=True):
    torch = d["torch"]
    g = torch.from_numpy(gs).cuda()
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    hits = torch.zeros((scenes.NUM_PMT,), dtype=torch.float64, device="cuda")
    grad = torch.zeros((scenes.NUM_PMT, 32), dtype=torch.float64, device="cuda")
    ADJ.adjoint_device(d["eng"], g, N, event, theta, d["mat_line"], *WL, hits, grad, pathwise=pathwise)
    torch.cuda.synchronize()
    return hits.cpu().numpy(), grad.cpu().numpy()


def test_adjoint_forward_equals_plain_engine(det):
    gs = scenes.detector_gensteps(4, 2000, seed=21, lib=det["lib"])
    hits, grad = _adj(det, gs, det["theta"], event=3)
    phys2 = ADJ.retabulate(det["phys"], det["theta"], det["mat_line"], *WL)
    eng2 = det["E"].Engine(det["fd"].arrays(), phys2, det["E"].default_config(max_photon=8000, num_sensor=scenes.NUM_PMT))
    r = eng2.simulate(gs, 3, sensor_hits=True)
    eng2.close()
    np.testing.assert_array_equal(hits.astype(np.int64), r["sensor_hits"].astype(np.int64))
    assert hits.sum() > 500


def test_adjoint_scores_match_fp64_cpu_estimator(det):
    gs = scenes.detector_gensteps(2, 1500, seed=22, lib=det["lib"])
    n = 3000
    hits, grad = _adj(det, gs, det["theta"], pathwise=False)    # the FP64 estimator holds the score terms
    phys2 = ADJ.retabulate(det["phys"], det["theta"], det["mat_line"], *WL)
    eng2 = det["E"].Engine(det["fd"].arrays(), phys2, det["E"].default_config(max_photon=n))
    u = eng2.rng_sequence(0, 0, n, 1024)
    eng2.close()
    S = O.Scene(det["fd"].arrays(), phys2)
    h64, g64, err = S.adjoint(gs, u, det["mat_line"], *WL, scenes.NUM_PMT)
    assert err & 1 == 0
    # same photons: identical hits, and score sums equal to float accumulation precision
    assert abs(h64.sum() - hits.sum()) <= 0.002 * hits.sum() + 2
    tot, tot64 = grad.sum(0), g64.sum(0)
    for kind in range(4):
        sl = slice(8 * kind, 8 * kind + 8)
        scale = np.abs(tot64[sl]).max()
        dev = np.abs(tot[sl] - tot64[sl]) / max(scale, 1e-30)
        print(ADJ.KINDS[kind], "engine", np.array2string(tot[sl], precision=4), "fp64", np.array2string(tot64[sl], precision=4),
              "max dev/scale", dev.max())
        # absorption / Rayleigh / reemission terms are sums of the same per-photon values: float vs double
        # accumulation only; the Fresnel (rindex) terms add float dual-number vs double derivatives
        assert dev.max() < (0.005 if kind < 3 else 0.05), ADJ.KINDS[kind]


def test_autograd_function_and_finite_differences(det):
    torch = det["torch"]
    M = 8                      # independent events give the standard errors of both estimators
    gs = scenes.detector_gensteps(10, 10000, seed=23, lib=det["lib"])
    g = torch.from_numpy(gs).cuda()
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    base = det["theta"].astype(np.float64)
    # autograd on one event: backward of sum(H) equals the summed Jacobian
    theta = torch.tensor(det["theta"], dtype=torch.float32, requires_grad=True)
    H = ADJ.expected_hits(theta, det["eng"], g, N, 0, det["mat_line"], *WL)
    H.sum().backward()
    _, J = _adj(det, gs, det["theta"], event=0)
    np.testing.assert_allclose(theta.grad.numpy(), J.sum(0), rtol=1e-5)
    ks = (3, 2, 4)             # absorption length in the bins holding the 430/20 nm emission
    adj, fd = {k: [] for k in ks}, {k: [] for k in ks}
    for ev in range(1, M + 1):
        _, Jev = _adj(det, gs, det["theta"], event=ev)
        for k in ks:
            h = 0.01 * base[k]
            tp, tm = base.copy(), base.copy()
            tp[k] += h
            tm[k] -= h
            hp, _ = _adj(det, gs, tp.astype(np.float32), event=ev)     # common random numbers: same event
            hm, _ = _adj(det, gs, tm.astype(np.float32), event=ev)
            fd[k].append((hp.sum() - hm.sum()) / (2 * h))
            adj[k].append(Jev[:, k].sum())
    for k in ks:
        a, f = np.array(adj[k]), np.array(fd[k])
        se = np.sqrt(a.var(ddof=1) / M + f.var(ddof=1) / M)
        z = (a.mean() - f.mean()) / se
        print(f"theta[{k}] adjoint {a.mean():.5g} +- {a.std(ddof=1)/np.sqrt(M):.2g}  fd {f.mean():.5g} +- "
              f"{f.std(ddof=1)/np.sqrt(M):.2g}  z {z:.2f}  rel {(a.mean()-f.mean())/f.mean():+.3f}")
        assert abs(z) < 4.0


@pytest.mark.parametrize("pool", [0, 1 << 12])
def test_adjoint_wavefront_equals_persistent(det, pool):
    """the adjoint pass in both loop forms: identical hits, score sums equal to float accumulation order;
    also through a 4,096-slot pool, whose refill rounds reload the score slots in slot order"""
    torch = det["torch"]
    gs = scenes.detector_gensteps(6, 3000, seed=31, lib=det["lib"])
    N = int(gs.view(np.int32)[:, 0, 3].sum())
    g = torch.from_numpy(gs).cuda()
    out = []
    for mode in (1, 2):
        eng = det["E"].Engine(det["fd"].arrays(), det["phys"],
                              det["E"].default_config(max_photon=N, num_sensor=scenes.NUM_PMT, kernel_mode=mode,
                                                      wave_pool=pool))
        h = torch.zeros((scenes.NUM_PMT,), dtype=torch.float64, device="cuda")
        j = torch.zeros((scenes.NUM_PMT, 32), dtype=torch.float64, device="cuda")
        ADJ.adjoint_device(eng, g, N, 2, det["theta"], det["mat_line"], *WL, h, j, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        out.append((h.cpu().numpy(), j.cpu().numpy()))
        eng.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][0].sum() > 500
    # per-photon scores agree to float rounding; the refractive-index terms are sums of large
    # cancelling Fresnel scores, so their totals agree to a relative 2e-3 of the term scale
    scale = np.abs(out[0][1]).sum(0) + 1e-12
    assert np.all(np.abs(out[0][1].sum(0) - out[1][1].sum(0)) <= 2e-3 * scale)


@pytest.mark.parametrize("rounds", [0, 2])
def test_adjoint_schedule_changes_no_result(det, rounds):
    """adj_wave_rounds (12 by default) against the 2-round schedule and the host-read one: identical
    hits, and score sums equal to float rounding (the adjoint step is inlined into the physics and
    the tail kernels, whose fast-math contractions differ in the last bits of the pathwise terms:
    about 1e-7 of a term's scale)"""
    gs = scenes.detector_gensteps(6, 3000, seed=33, lib=det["lib"])
    h0, j0 = _adj(det, gs, det["theta"], event=4)
    eng = det["eng"]
    default = int(eng.config.adj_wave_rounds)
    assert default == int(det["E"].default_config().adj_wave_rounds) and default != rounds
    try:
        eng.set_launch_config(adj_wave_rounds=rounds)
        h1, j1 = _adj(det, gs, det["theta"], event=4)
        assert eng.last_call_stats()["wave_rounds"] >= (rounds if rounds else 1)
    finally:
        eng.set_launch_config(adj_wave_rounds=default)
    np.testing.assert_array_equal(h0, h1)
    assert h0.sum() > 500
    scale = np.abs(j0).sum(0) + 1e-12
    assert np.all(np.abs(j0.sum(0) - j1.sum(0)) <= 1e-5 * scale)


def test_refractive_index_gradient_with_pathwise_term(det):
    """d(total hits)/d n in the bin holding the emission peak (420-460 nm): the pathwise tangent of the
    refracted direction carries most of it (the Fresnel score alone is a few per cent of it); the
    adjoint agrees with central differences (step 1e-3 relative, common random numbers)"""
    M = 48
    gs = scenes.detector_gensteps(50, 10000, seed=29, lib=det["lib"])
    base = det["theta"].astype(np.float64)
    k = 27
    h = 1e-3 * base[k]
    adj, adj0, fd = [], [], []
    for ev in range(1, M + 1):
        adj.append(_adj(det, gs, det["theta"], event=ev)[1][:, k].sum())
        adj0.append(_adj(det, gs, det["theta"], event=ev, pathwise=False)[1][:, k].sum())
        tp, tm = base.copy(), base.copy()
        tp[k] += h
        tm[k] -= h
        fd.append((_adj(det, gs, tp.astype(np.float32), event=ev)[0].sum() -
                   _adj(det, gs, tm.astype(np.float32), event=ev)[0].sum()) / (2 * h))
    a, a0, f = np.array(adj), np.array(adj0), np.array(fd)
    se = np.sqrt(a.var(ddof=1) / M + f.var(ddof=1) / M)
    z = (a.mean() - f.mean()) / se
    print(f"rindex bin 3: adjoint {a.mean():.1f} +- {a.std(ddof=1)/np.sqrt(M):.1f} (score only {a0.mean():.1f}) "
          f"fd {f.mean():.1f} +- {f.std(ddof=1)/np.sqrt(M):.1f}  z {z:.2f}")
    assert f.mean() < 0 and abs(a0.mean()) < 0.3 * abs(f.mean())    # the score alone misses it
    assert abs(z) < 4.0
