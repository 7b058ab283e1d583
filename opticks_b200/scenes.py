"""Synthetic workloads: geometry, properties and gensteps with the shapes of the benchmark
configurations.  All randomness is numpy PCG64 with explicit seeds.

* ``sphere_in_box``  : 1 m water sphere (n 1.333, absorption 10 m, Rayleigh 5 m) in a 3 m vacuum
  box whose inner surface detects with efficiency 1; one torch genstep at the origin.
* ``csg_scan_tree``  : ((cyl r250 h400 U zsph r254 z[0,190]) - (sph r240 ^ box 500x500x300)) U
  torus(R200, r20) at z=-200, as one 15-node complete tree; rays uniform in a 2 m cube.
* ``detector``       : LS sphere r 17.7 m inside a 120 mm acrylic shell inside a water sphere
  r 20.5 m, 17,612 PMT-like instances (zsphere cap r254 U cylinder neck r50 h200) on a
  Fibonacci lattice at r 19.4 m facing inward, cap surface detect 0.3 / absorb 0.7;
  scintillation gensteps with vertices uniform in r < 17 m and a Gaussian 430/20 nm spectrum.
"""
from __future__ import annotations

import math

import numpy as np

from . import foundry as F
from . import material as M

GS_TORCH = 6
GS_SCINTILLATION = 16
GS_CERENKOV = 15
GS_CARRIER = 14
GS_INPUT_PHOTON = 19
T_SPHERE = 7
T_SPHERE_RANDPOL = 64    # T_SPHERE with a random linear polarisation (one extra uniform)
T_POINT = 3
T_DISC = 1

WATER_C1 = M.Material("Water", rindex=1.333, absorption_length=10000.0, scattering_length=5000.0)
VACUUM = M.Material("Vacuum", rindex=1.0, absorption_length=1e9, scattering_length=1e9)


def torch_genstep(numphoton: int, pos=(0.0, 0.0, 0.0), wavelength=440.0, radius=0.0, type_=T_SPHERE_RANDPOL,
                  mom=(0.0, 0.0, 1.0), time=0.0, zenith=(0.0, 1.0), azimuth=(0.0, 1.0), distance=0.0) -> np.ndarray:
    """quad6 storch (sysrap/storch.h:43-80)"""
    g = np.zeros((6, 4), dtype=np.float32)
    gi = g.view(np.int32)
    gi[0] = (GS_TORCH, 0, 0, numphoton)
    g[1] = (*pos, time)
    m = np.asarray(mom, dtype=np.float64)
    m = m / np.linalg.norm(m)
    g[2] = (*m, 1.0)
    g[3] = (0.0, 0.0, 1.0, wavelength)
    g[4] = (*zenith, *azimuth)
    g[5, 0] = radius
    g[5, 1] = distance
    gi[5, 2] = 0
    gi[5, 3] = type_
    return g


def input_photon_genstep(num_photon: int) -> np.ndarray:
    """SEvent::MakeInputPhotonGenstep (sysrap/SEvent.cc:120-133): gencode INPUT_PHOTON and the photon
    count; the photons themselves are set on the engine (Engine.set_input_photon)"""
    g = np.zeros((6, 4), dtype=np.float32)
    g.view(np.int32)[0] = (GS_INPUT_PHOTON, 0, 0, num_photon)
    return g


def carrier_genstep(numphoton: int, pos=(0.0, 0.0, 0.0), time=0.0, mom=(1.0, 0.0, 0.0), pol=(0.0, 1.0, 0.0),
                    wavelength=500.0) -> np.ndarray:
    """scarrier (sysrap/scarrier.h): rows 2-5 are the photon itself (moved 10 mm in y per photon)"""
    g = np.zeros((6, 4), dtype=np.float32)
    g.view(np.int32)[0] = (GS_CARRIER, 0, 0, numphoton)
    g[2] = (*pos, time)
    g[3, :3] = mom
    g[4] = (*pol, wavelength)
    return g


def input_photons(n: int, seed: int = 0, radius: float = 100.0, wavelength: float = 440.0) -> np.ndarray:
    """(n,4,4) sphoton rows: positions in a ball, isotropic directions, transverse polarisations"""
    rng = np.random.default_rng(seed)
    p = np.zeros((n, 4, 4), np.float32)
    p[:, 0, :3] = uniform_ball(n, radius, rng)
    p[:, 0, 3] = rng.uniform(0.0, 1.0, n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    t = np.cross(d, rng.normal(size=(n, 3)))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    p[:, 1, :3] = d
    p[:, 2, :3] = t
    p[:, 2, 3] = wavelength
    return p


def scint_genstep(numphoton: int, pos, matline: int, time=0.0, delta=(0.0, 0.0, 1.0), step_length=1.0,
                  charge=1.0, mean_velocity=250.0, scint_time=5.0) -> np.ndarray:
    """quad6 sscint (sysrap/sscint.h:34-74)"""
    g = np.zeros((6, 4), dtype=np.float32)
    gi = g.view(np.int32)
    gi[0] = (GS_SCINTILLATION, 0, matline, numphoton)
    g[1] = (*pos, time)
    g[2] = (*delta, step_length)
    gi[3, 0] = 0
    g[3, 1:] = (charge, 1.0, mean_velocity)
    g[5, 0] = scint_time
    return g


def cerenkov_genstep(numphoton: int, pos, matline: int, delta=(0.0, 0.0, 10.0), beta_inverse=1.0 / 0.99,
                     wmin=300.0, wmax=600.0, nmax=1.5, pre_velocity=296.8, post_velocity=296.5, time=0.0) -> np.ndarray:
    """quad6 scerenkov (sysrap/scerenkov.h:29-60)"""
    g = np.zeros((6, 4), dtype=np.float32)
    gi = g.view(np.int32)
    gi[0] = (GS_CERENKOV, 0, matline, numphoton)
    g[1] = (*pos, time)
    step = float(np.linalg.norm(delta))
    g[2] = (*delta, step)
    gi[3, 0] = 0
    g[3, 1:] = (1.0, 1.0, pre_velocity)
    max_cos = beta_inverse / nmax
    max_sin2 = (1.0 - max_cos) * (1.0 + max_cos)
    g[4] = (beta_inverse, wmin, wmax, max_cos)
    g[5] = (max_sin2, float(numphoton), float(numphoton), post_velocity)
    return g


# ---------------------------------------------------------------- C1
def sphere_in_box(num_photon: int = 1_000_000):
    lib = M.BoundaryLib()
    lib.mat(VACUUM)
    lib.mat(M.Material("Rock", rindex=1.5, absorption_length=1.0, scattering_length=1e9))
    lib.mat(WATER_C1)
    lib.sur(M.Surface("Detector", detect=1.0, absorb=0.0))
    b_box = lib.add("Rock", "", "Detector", "Vacuum")
    b_sph = lib.add("Vacuum", "", "", "Water")
    fd = F.Foundry()
    p0 = fd.add_prim(F.box3(3000.0, 3000.0, 3000.0), b_box)
    p1 = fd.add_prim(F.sphere(1000.0), b_sph)
    s0 = fd.add_solid("box_sphere", [p0, p1])
    fd.add_inst(np.eye(4), s0)
    gs = torch_genstep(num_photon, wavelength=440.0, radius=0.0, type_=T_SPHERE_RANDPOL)[None]
    return fd, lib, None, gs


def sphere_in_box_surface(num_photon: int = 200_000, detect: float = 0.2, absorb: float = 0.2,
                          reflect_specular: float = 0.3, reflect_diffuse: float = 0.3):
    """C1's sphere-in-box with a box surface that also reflects: each wall hit detects, absorbs,
    reflects diffusely (Lambertian) or specularly with the given fractions, so photons cross the
    box and the water sphere many times (qudarap/qsim.h:1680-1750 picks the branch with one
    uniform; the specular share is what is left over, qsim.h never reads reflect_specular)"""
    lib = M.BoundaryLib()
    lib.mat(VACUUM)
    lib.mat(M.Material("Rock", rindex=1.5, absorption_length=1.0, scattering_length=1e9))
    lib.mat(WATER_C1)
    lib.sur(M.Surface("Wall", detect=detect, absorb=absorb, reflect_specular=reflect_specular,
                      reflect_diffuse=reflect_diffuse))
    b_box = lib.add("Rock", "", "Wall", "Vacuum")
    b_sph = lib.add("Vacuum", "", "", "Water")
    fd = F.Foundry()
    p0 = fd.add_prim(F.box3(3000.0, 3000.0, 3000.0), b_box)
    p1 = fd.add_prim(F.sphere(1000.0), b_sph)
    s0 = fd.add_solid("box_sphere", [p0, p1])
    fd.add_inst(np.eye(4), s0)
    gs = torch_genstep(num_photon, wavelength=440.0, radius=0.0, type_=T_SPHERE, distance=0.25)[None]
    return fd, lib, None, gs


# ---------------------------------------------------------------- C2
def csg_scan_tree(with_torus: bool = True):
    """returns (foundry, prim index) of the 15-node tree"""
    cyl = F.cylinder(250.0, -200.0, 200.0)
    zs = F.zsphere(254.0, 0.0, 190.0)
    sp = F.sphere(240.0)
    bx = F.box3(500.0, 500.0, 300.0)
    left = F.op("difference", F.op("union", cyl, zs), F.op("intersection", sp, bx))
    if with_torus:
        tor = F.translate(F.torus(200.0, 20.0), 0.0, 0.0, -200.0)
        root = F.op("union", left, tor)
    else:
        root = left
    fd = F.Foundry()
    p = fd.add_prim(root, 0)
    s = fd.add_solid("scan", [p])
    fd.add_inst(np.eye(4), s)
    return fd, p


# zoo prims whose trees hold a slab, infcylinder or disc leaf: the reference compiles those three
# leaves only under CSG_EXTRA (CSG/csg_intersect_leaf.h:100-108,224-232), so its tree intersector
# misses them; they are compared leaf by leaf against the reference's leaf functions instead
ZOO_EXTRA_PRIMS = (8, 9, 10, 13)


def csg_leaf_zoo():
    """(foundry, prim indices) exercising the cone, hyperboloid, convexpolyhedron, phicut,
    halfspace, slab, infcylinder and disc leaves alone, transformed, complemented and inside small
    trees (unbounded leaves always cut by a bounded one)"""
    octa = [(sx / math.sqrt(3.0), sy / math.sqrt(3.0), sz / math.sqrt(3.0), 180.0)
            for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)]
    comp_phi = F.phicut(0.5, 2.0)
    comp_phi.complement = True
    trees = [
        F.cone(200.0, -150.0, 50.0, 150.0),
        F.translate(F.cone(80.0, -100.0, 220.0, 120.0), 30.0, -40.0, 20.0),
        F.hyperboloid(150.0, 120.0, -200.0, 200.0),
        F.convexpolyhedron(F.cube_planes(150.0), (-150, -150, -150, 150, 150, 150)),
        F.convexpolyhedron(octa, (-312, -312, -312, 312, 312, 312)),
        F.op("intersection", F.sphere(250.0), F.phicut(0.3, 2.5)),
        F.op("intersection", F.cylinder(250.0, -200.0, 200.0), F.phicut(-1.0, 3.5)),
        F.op("intersection", F.sphere(250.0), F.halfspace((0.0, 0.0, 1.0), 50.0)),
        F.op("intersection", F.box3(500.0, 500.0, 500.0), F.slab((0.6, 0.8, 0.0), -100.0, 150.0)),
        F.op("intersection", F.infcylinder(120.0), F.box3(600.0, 600.0, 400.0)),
        F.disc(50.0, 250.0, -10.0, 10.0),
        F.op("difference", F.cone(220.0, -200.0, 20.0, 200.0), F.convexpolyhedron(F.cube_planes(90.0), (-90, -90, -90, 90, 90, 90))),
        F.op("intersection", F.sphere(240.0), comp_phi),
        F.op("union", F.hyperboloid(100.0, 80.0, -150.0, 150.0), F.disc(0.0, 230.0, -5.0, 5.0)),
    ]
    fd = F.Foundry()
    prims = [fd.add_prim(t, 0) for t in trees]
    fd.add_solid("zoo", prims)
    fd.add_inst(np.eye(4), 0)
    return fd, prims


def csg_list_zoo():
    """(foundry, prim indices) of list nodes: contiguous, discontiguous and overlap lists of
    spheres, boxes, cylinders and a convexpolyhedron (translated leaves), and lists as leaves of
    boolean trees.  No contiguous list puts more than 8 enters on one ray."""
    def sph(r, x, y, z=0.0):
        return F.translate(F.sphere(r), x, y, z)
    s2 = 100.0 * math.sqrt(2.0)
    three = lambda r: [sph(r, 100.0, 100.0), sph(r, -100.0, 100.0), sph(r, 0.0, -s2)]
    cube = F.convexpolyhedron(F.cube_planes(60.0), (-60, -60, -60, 60, 60, 60))
    chain = [F.translate(F.cylinder(40.0, -60.0, 60.0), 0.0, 0.0, z) for z in (-200.0, -100.0, 0.0, 100.0, 200.0)]
    trees = [
        F.list_node("contiguous", three(150.0)),
        F.list_node("discontiguous", three(80.0)),
        F.list_node("overlap", [F.box3(300.0, 300.0, 300.0), F.sphere(200.0)]),
        F.list_node("overlap", three(260.0)),
        F.list_node("contiguous", [F.box3(300.0, 300.0, 300.0), F.sphere(200.0)]),
        F.list_node("discontiguous", [sph(60.0, -50.0, 0.0), sph(60.0, 50.0, 0.0),
                                      F.translate(F.box3(80.0, 80.0, 80.0), 0.0, 200.0, 0.0),
                                      F.translate(F.box3(80.0, 80.0, 80.0), 0.0, -200.0, 0.0)]),
        F.op("union", F.box3(200.0, 200.0, 200.0), F.list_node("contiguous", three(120.0))),
        F.op("difference", F.list_node("contiguous", three(150.0)), F.sphere(120.0)),
        F.list_node("discontiguous", [F.translate(cube, 150.0, 0.0, 0.0), sph(70.0, -150.0, 0.0)]),
        F.list_node("contiguous", chain),
        F.op("intersection", F.list_node("overlap", [F.box3(300.0, 300.0, 300.0), F.sphere(200.0)]),
             F.list_node("discontiguous", [sph(90.0, 0.0, 120.0), sph(90.0, 0.0, -120.0)])),
    ]
    fd = F.Foundry()
    prims = [fd.add_prim(t, 0) for t in trees]
    fd.add_solid("lists", prims)
    fd.add_inst(np.eye(4), 0)
    return fd, prims


def leaf_zoo_detector(num_photon: int = 100_000):
    """photons from the centre of a water-filled box whose walls detect, through acrylic bodies
    made of the further leaves: a cone, a hyperboloid, an octahedral convexpolyhedron, a sphere cut
    by a phicut wedge, a sphere cut by a halfspace and a cone minus a convexpolyhedron cube"""
    lib = M.BoundaryLib()
    lib.mat(VACUUM)
    lib.mat(M.Material("Rock", rindex=1.5, absorption_length=1.0, scattering_length=1e9))
    lib.mat(WATER_C1)
    lib.mat(M.Material("Acrylic", rindex=1.49, absorption_length=1e6, scattering_length=1e6))
    lib.sur(M.Surface("Detector", detect=1.0, absorb=0.0))
    b_box = lib.add("Rock", "", "Detector", "Water")
    b_acr = lib.add("Water", "", "", "Acrylic")
    octa = [(sx / math.sqrt(3.0), sy / math.sqrt(3.0), sz / math.sqrt(3.0), 180.0)
            for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)]
    bodies = [
        F.translate(F.cone(200.0, -150.0, 50.0, 150.0), 800.0, 0.0, 0.0),
        F.translate(F.hyperboloid(120.0, 100.0, -200.0, 200.0), -800.0, 0.0, 0.0),
        F.translate(F.convexpolyhedron(octa, (-312, -312, -312, 312, 312, 312)), 0.0, 800.0, 0.0),
        F.translate(F.op("intersection", F.sphere(250.0), F.phicut(0.3, 2.5)), 0.0, -800.0, 0.0),
        F.translate(F.op("intersection", F.sphere(250.0), F.halfspace((0.0, 0.0, 1.0), 50.0)), 0.0, 0.0, 800.0),
        F.translate(F.op("difference", F.cone(220.0, -200.0, 20.0, 200.0),
                         F.convexpolyhedron(F.cube_planes(90.0), (-90, -90, -90, 90, 90, 90))), 0.0, 0.0, -800.0),
    ]
    fd = F.Foundry()
    prims = [fd.add_prim(F.box3(3000.0, 3000.0, 3000.0), b_box)] + [fd.add_prim(b, b_acr) for b in bodies]
    s0 = fd.add_solid("zoo", prims)
    fd.add_inst(np.eye(4), s0)
    gs = torch_genstep(num_photon, wavelength=440.0, radius=0.0, type_=T_SPHERE, distance=0.25)[None]
    return fd, lib, None, gs


def list_zoo_detector(num_photon: int = 100_000):
    """photons from the centre of a water-filled box whose walls detect, through acrylic bodies
    that are list nodes (contiguous, discontiguous, overlap) and trees holding lists"""
    lib = M.BoundaryLib()
    lib.mat(VACUUM)
    lib.mat(M.Material("Rock", rindex=1.5, absorption_length=1.0, scattering_length=1e9))
    lib.mat(WATER_C1)
    lib.mat(M.Material("Acrylic", rindex=1.49, absorption_length=1e6, scattering_length=1e6))
    lib.sur(M.Surface("Detector", detect=1.0, absorb=0.0))
    b_box = lib.add("Rock", "", "Detector", "Water")
    b_acr = lib.add("Water", "", "", "Acrylic")

    def sph(r, x, y, z=0.0):
        return F.translate(F.sphere(r), x, y, z)
    s2 = 100.0 * math.sqrt(2.0)
    three = lambda r: [sph(r, 100.0, 100.0), sph(r, -100.0, 100.0), sph(r, 0.0, -s2)]
    bodies = [
        F.translate(F.list_node("contiguous", three(150.0)), 900.0, 0.0, 0.0),
        F.translate(F.list_node("discontiguous", three(80.0)), -900.0, 0.0, 0.0),
        F.translate(F.list_node("overlap", [F.box3(300.0, 300.0, 300.0), F.sphere(200.0)]), 0.0, 900.0, 0.0),
        F.translate(F.list_node("contiguous", [F.box3(300.0, 300.0, 300.0), F.sphere(200.0)]), 0.0, -900.0, 0.0),
        F.translate(F.op("union", F.box3(200.0, 200.0, 200.0), F.list_node("contiguous", three(120.0))), 0.0, 0.0, 900.0),
        F.translate(F.op("difference", F.list_node("contiguous", three(150.0)), F.sphere(120.0)), 0.0, 0.0, -900.0),
    ]
    fd = F.Foundry()
    prims = [fd.add_prim(F.box3(3000.0, 3000.0, 3000.0), b_box)] + [fd.add_prim(b, b_acr) for b in bodies]
    s0 = fd.add_solid("lists", prims)
    fd.add_inst(np.eye(4), s0)
    gs = torch_genstep(num_photon, wavelength=440.0, radius=0.0, type_=T_SPHERE, distance=0.25)[None]
    return fd, lib, None, gs


def scan_rays(n: int, seed: int = 0, half: float = 1000.0) -> np.ndarray:
    """(6,n) SoA: origins uniform in a 2 m cube, directions uniform on the sphere"""
    rng = np.random.Generator(np.random.PCG64(seed))
    o = rng.uniform(-half, half, size=(3, n))
    ct = rng.uniform(-1.0, 1.0, size=n)
    ph = rng.uniform(0.0, 2 * math.pi, size=n)
    st = np.sqrt(1.0 - ct * ct)
    d = np.stack([st * np.cos(ph), st * np.sin(ph), ct])
    return np.ascontiguousarray(np.concatenate([o, d]).astype(np.float32))


# ---------------------------------------------------------------- C3/C4/C5
R_LS, T_ACRYLIC, R_WATER, R_PMT = 17700.0, 120.0, 20500.0, 19400.0
NUM_PMT = 17612


def ls_rindex(wl):
    wl = np.asarray(wl, dtype=np.float64)
    return np.clip(1.50 + (wl - 300.0) * (1.48 - 1.50) / 300.0, 1.44, 1.56)


def detector_lib(pmt_ems: int = M.EMS_SURFACE, world_surface: M.Surface | None = None):
    """the detector's boundary library.  ``pmt_ems`` is the PMT cathode's surface kind: with
    ``EMS_SENSOR_A`` (smatsur_Surface_zplus_sensor_A) a hit on the PMT's upper hemisphere (local
    z >= 0) always detects and one below it takes the ordinary surface branch (qudarap/qsim.h:
    2304-2316).  ``world_surface`` replaces the absorbing rock surface, e.g. with a reflecting one
    so that photons come back onto the backs of the PMTs."""
    lib = M.BoundaryLib()
    ls = M.Material("LS", rindex=ls_rindex, absorption_length=60000.0, scattering_length=27000.0,
                    reemission_prob=lambda wl: np.where(np.asarray(wl) < 400.0, 0.5, 0.0))
    acr = M.Material("Acrylic", rindex=1.49, absorption_length=1e6, scattering_length=1e6)
    water = M.Material("Water", rindex=1.333, absorption_length=40000.0, scattering_length=50000.0)
    rock = M.Material("Rock", rindex=1.5, absorption_length=1.0, scattering_length=1e9)
    pyrex = M.Material("Pyrex", rindex=1.458, absorption_length=1e3, scattering_length=1e9)
    for m in (ls, acr, water, rock, pyrex):
        lib.mat(m)
    world = world_surface or M.Surface("RockAbsorber", detect=0.0, absorb=1.0)
    lib.sur(world)
    lib.sur(M.Surface("PMTCathode", detect=0.3, absorb=0.7, ems=pmt_ems))
    b_world = lib.add("Rock", "", world.name, "Water")
    b_acr = lib.add("Water", "", "", "Acrylic")
    b_ls = lib.add("Acrylic", "", "", "LS")
    b_pmt = lib.add("Water", "PMTCathode", "PMTCathode", "Pyrex")
    return lib, (b_world, b_acr, b_ls, b_pmt)


def detector(num_pmt: int = NUM_PMT, pmt_ems: int = M.EMS_SURFACE, world_surface: M.Surface | None = None):
    lib, (b_world, b_acr, b_ls, b_pmt) = detector_lib(pmt_ems, world_surface)
    fd = F.Foundry()
    p_world = fd.add_prim(F.sphere(R_WATER), b_world)
    p_acr = fd.add_prim(F.sphere(R_LS + T_ACRYLIC), b_acr)
    p_ls = fd.add_prim(F.sphere(R_LS), b_ls)
    s0 = fd.add_solid("global", [p_world, p_acr, p_ls])
    pmt = F.op("union", F.zsphere(254.0, 0.0, 190.0), F.cylinder(50.0, -200.0, 0.0))
    p_pmt = fd.add_prim(pmt, b_pmt)
    s1 = fd.add_solid("pmt", [p_pmt])
    fd.add_inst(np.eye(4), s0)
    for i, pos in enumerate(F.fibonacci_sphere(num_pmt, R_PMT)):
        fd.add_inst(F.look_at_z(pos, (0.0, 0.0, 0.0)), s1, sensor_identifier=i, sensor_index=i)
    icdf = M.gaussian_icdf(430.0, 20.0)
    return fd, lib, icdf


def uniform_ball(n: int, radius: float, rng) -> np.ndarray:
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    r = radius * rng.uniform(0.0, 1.0, size=n) ** (1.0 / 3.0)
    return v * r[:, None]


def detector_gensteps(num_genstep: int = 1000, photons_per_genstep: int = 10000, seed: int = 0, lib=None) -> np.ndarray:
    if lib is None:
        lib, _ = detector_lib()
    matline = lib.material_line("LS")
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = uniform_ball(num_genstep, 17000.0, rng)
    dirs = rng.normal(size=(num_genstep, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    return np.stack([scint_genstep(photons_per_genstep, pos[i], matline, delta=tuple(dirs[i]), step_length=1.0)
                     for i in range(num_genstep)])


def batched_events(num_event: int = 4096, median: float = 50000.0, sigma_ln: float = 1.0,
                   lo: int = 1000, hi: int = 5_000_000, lib=None):
    """one scintillation genstep per event; count lognormal, vertex uniform r<17 m, seeded by event"""
    if lib is None:
        lib, _ = detector_lib()
    matline = lib.material_line("LS")
    gs = []
    for ev in range(num_event):
        rng = np.random.Generator(np.random.PCG64(ev))
        n = int(np.clip(round(median * math.exp(sigma_ln * rng.normal())), lo, hi))
        pos = uniform_ball(1, 17000.0, rng)[0]
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        gs.append(scint_genstep(n, pos, matline, delta=tuple(d)))
    return np.stack(gs)
