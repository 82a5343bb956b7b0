"""Parity of the CUDA step (through the C-ABI) with the oracle and the goldens.

Metric: per field, max|gpu - ref| / max|ref| after N steps.  The tolerance
of each field is the larger of the stated target 1e-5 and TOL_FACTOR times
the FP32 round-off floor of the same case (the oracle in float against the
oracle in double), because two FP32 implementations of this step cannot
agree more closely than their own round-off: the non-equilibrium moments
Pi^neq are a ~1e-4 remainder of O(1) population sums.
"""
import numpy as np
import pytest

from entropicthreadsafe_b200 import capi, workloads
from helpers import (GOLDEN_CASES, field_errors, golden_inlet, golden_params, load_golden, rel_err, run_gpu,
                     run_oracle, with_halo)

pytestmark = pytest.mark.gpu

TARGET = 1e-5      # max relative error per field (stated target)
TOL_FACTOR = 4.0   # allowed multiple of the FP32 round-off floor


def assert_parity(gpu, o64, o32, label):
    eg = field_errors(gpu, o64)
    e32 = field_errors(o32, o64)
    bad = {k: (eg[k], e32[k]) for k in eg if eg[k] > max(TARGET, TOL_FACTOR * e32[k])}
    assert not bad, f"{label}: field: (gpu err, fp32 floor) {bad}"
    return eg, e32


@pytest.mark.parametrize("case", GOLDEN_CASES)
def test_golden_through_capi(case):
    """Reference statements (golden) -> populations -> tslb_upload_pops -> steps."""
    from entropicthreadsafe_b200.solver import Lattice
    d, meta = load_golden(case)
    nz, ny, nx = d["rho_fp64"].shape
    with Lattice(golden_params(meta), nx, ny, nz) as lat:
        for face, planes in (golden_inlet(d) or {}).items():
            lat.set_inlet(face, planes)
        lat.upload_pops(with_halo(d["f_fp32"]), with_halo(d["g_fp32"]))
        lat.step(meta["nsteps"])
        out = lat.download()
    ref64 = {k: d[k + "_fp64"] for k in capi.FIELDS}
    ref32 = {k: d[k + "_fp32"] for k in capi.FIELDS}
    assert_parity(out, ref64, ref32, case)


def small_droplet(n=24, R=6.0):
    p, f = workloads.droplet(n=n, radius=R, tau=0.8, sigma=0.01, beta=0.7)
    return p, f


def test_colour_droplet_100_steps():
    p, f = small_droplet()
    gpu, _ = run_gpu(p, f, 100)
    o64, _ = run_oracle(p, f, 100, fp64=True)
    o32, _ = run_oracle(p, f, 100, fp64=False)
    assert_parity(gpu, o64, o32, "colour droplet")


def test_colour_channel_walls_force_100_steps():
    p, f = workloads.channel(nx=40, ny=24, nz=20, ndrops=3, radius=4.0, wall_gap=2.0, gx=2.5e-5)
    gpu, _ = run_gpu(p, f, 100)
    o64, _ = run_oracle(p, f, 100, fp64=True)
    o32, _ = run_oracle(p, f, 100, fp64=False)
    assert_parity(gpu, o64, o32, "colour channel")


def test_colour_moving_walls_viscosity_ratio():
    p, f = small_droplet(n=24, R=5.0)
    p.tau_b = 1.1
    for face, u in ((capi.FACE_ZM, -0.05), (capi.FACE_ZP, 0.05)):
        p.bc[face] = capi.BC_VELOCITY
        p.bc_u[face][0] = u
        p.bc_phi[face] = -1.0
    p.wall_phi_mode = 1
    gpu, _ = run_gpu(p, f, 60)
    o64, _ = run_oracle(p, f, 60, fp64=True)
    o32, _ = run_oracle(p, f, 60, fp64=False)
    assert_parity(gpu, o64, o32, "colour Couette")


def test_phasefield_jet_inlet_outlet():
    n, nz = 20, 24
    p = capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=0.6, sigma=0.01, sharp_c=0.9,
                         bc=[capi.BC_PERIODIC] * 4 + [capi.BC_INLET, capi.BC_OUTLET],
                         bc_u=[[0, 0, 0]] * 5 + [[0, 0, 0.05]], bc_phi=[0.0] * 6, wall_phi_mode=0)
    f = workloads.empty_fields(n, n, nz)
    y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    disc = ((x - n / 2) ** 2 + (y - n / 2) ** 2 <= 4.0 ** 2)
    planes = np.zeros((4, n, n), np.float32)
    planes[2] = np.where(disc, 0.05, 0.0)
    planes[3] = np.where(disc, 1.0, 0.0)
    inlet = {capi.FACE_ZM: planes}
    gpu, _ = run_gpu(p, f, 80, inlet=inlet)
    o64, _ = run_oracle(p, f, 80, fp64=True, inlet=inlet)
    o32, _ = run_oracle(p, f, 80, fp64=False, inlet=inlet)
    assert_parity(gpu, o64, o32, "phase-field jet")


def test_colour_jet_inlet_pressure_outlet():
    """Colour jet: device-drawn disc inlet at z-, pressure outlet at z+."""
    p, f, spec = workloads.jet(1, nx=20, ny=18, nz=24, diameter=6.0, nu=0.02)
    planes = workloads.inlet_disc(20, 18, 2, 1.0, spec["cx"], spec["cy"], 3.0, spec["w_in"], spec["noise"], 9, 0)
    inlet = {capi.FACE_ZM: planes}
    gpu, _ = run_gpu(p, f, 80, inlet=inlet)
    o64, _ = run_oracle(p, f, 80, fp64=True, inlet=inlet)
    o32, _ = run_oracle(p, f, 80, fp64=False, inlet=inlet)
    assert_parity(gpu, o64, o32, "colour jet, pressure outlet")
    # the pressure outlet holds the outlet density near 1
    assert abs(float(np.mean(o64["rho"][-1])) - 1.0) < 2e-3


def single_component_case(nx, ny, nz, seed, bc, bc_u, force):
    rng = np.random.default_rng(seed)
    # sigma = 0: the oracle's phase-field step then has no CSF force whatever its
    # phi does at the walls, and its f step is fused_TSLB_force_1c
    p = capi.make_params(mode=capi.MODE_SINGLE, tau_a=0.6, sigma=0.0, force=force, bc=bc, bc_u=bc_u)
    f = workloads.empty_fields(nx, ny, nz)
    for k in ("u", "v", "w"):
        f[k][:] = rng.normal(0, 0.02, f[k].shape)
    for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        f[k][:] = rng.normal(0, 1e-4, f[k].shape)
    f["rho"][:] = 1.0 + rng.normal(0, 1e-3, f["rho"].shape)
    f["phi"][:] = 1.0
    return p, f


@pytest.mark.parametrize("walls", ["periodic", "bounceback_and_moving_wall"])
def test_single_component_matches_oracle(walls):
    """Single-component mode against the phase-field oracle at sigma = 0,
    whose f step is the reference's fused_TSLB_force_1c."""
    if walls == "periodic":
        bc, bcu = [capi.BC_PERIODIC] * 6, [[0, 0, 0]] * 6
    else:
        bc = [capi.BC_PERIODIC] * 4 + [capi.BC_BOUNCEBACK, capi.BC_VELOCITY]
        bcu = [[0, 0, 0]] * 5 + [[0.03, 0.0, 0.0]]
    p, f = single_component_case(20, 18, 24, 3, bc, bcu, (1e-5, 2e-6, 0.0))
    gpu, _ = run_gpu(p, f, 100)
    o64, _ = run_oracle(p, f, 100, fp64=True)
    o32, _ = run_oracle(p, f, 100, fp64=False)
    assert np.all(gpu["phi"] == 1.0)
    for k in ("phi",):
        gpu.pop(k); o64.pop(k); o32.pop(k)
    eg = {k: rel_err(gpu[k], o64[k]) for k in gpu}
    e32 = {k: rel_err(o32[k], o64[k]) for k in gpu}
    bad = {k: (eg[k], e32[k]) for k in eg if eg[k] > max(TARGET, TOL_FACTOR * e32[k])}
    assert not bad, bad


def test_phasefield_droplet_bounceback_all_faces():
    n = 20
    p = capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=0.7, sigma=0.01, sharp_c=0.9,
                         force=(1e-5, 0.0, -2e-5), bc=[capi.BC_BOUNCEBACK] * 6, bc_phi=[0.0] * 6)
    f = workloads.empty_fields(n, n, n)
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    r = np.sqrt((x - 9.5) ** 2 + (y - 9.5) ** 2 + (z - 9.5) ** 2)
    f["phi"][:] = 0.5 * (1 + np.tanh((5 - r) / 1.5))
    gpu, _ = run_gpu(p, f, 60)
    o64, _ = run_oracle(p, f, 60, fp64=True)
    o32, _ = run_oracle(p, f, 60, fp64=False)
    assert_parity(gpu, o64, o32, "phase-field box")


def test_odd_sizes_partial_tiles():
    """Sizes that are not multiples of the 32x8 tile, periodic."""
    p, f = workloads.droplet(n=24, radius=6.0)
    # crop to an odd box
    f = {k: np.ascontiguousarray(v[:19, :13, :23]) for k, v in f.items()}
    gpu, _ = run_gpu(p, f, 30)
    o64, _ = run_oracle(p, f, 30, fp64=True)
    o32, _ = run_oracle(p, f, 30, fp64=False)
    assert_parity(gpu, o64, o32, "odd sizes")


@pytest.mark.parametrize("walls", ["periodic", "bounceback_xy"])
def test_row_staging_partial_tiles(walls):
    """nx = 44, a multiple of the 16-byte chunk: planes are staged in 16-byte
    chunks.  The second x tile is partial; with periodic faces its staged rows
    wrap around the x faces, with walls the chunks behind the x and y faces are
    ghost values."""
    p, _ = workloads.droplet(n=24, radius=5.0)
    nx, ny, nz = 44, 12, 16
    f = workloads.empty_fields(nx, ny, nz)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    # a droplet across the boundary of the two x tiles, and velocity noise
    r = np.sqrt((x - 31.5) ** 2 + (y - 5.5) ** 2 + (z - 7.5) ** 2)
    f["phi"][:] = np.tanh((4.5 - r) / 1.5)
    rng = np.random.default_rng(5)
    for k in ("u", "v", "w"):
        f[k][:] = rng.normal(0.0, 0.01, f[k].shape)
    if walls != "periodic":
        for face in (capi.FACE_XM, capi.FACE_XP, capi.FACE_YM, capi.FACE_YP):
            p.bc[face] = capi.BC_BOUNCEBACK
            p.bc_phi[face] = -1.0
    gpu, _ = run_gpu(p, f, 30)
    o64, _ = run_oracle(p, f, 30, fp64=True)
    o32, _ = run_oracle(p, f, 30, fp64=False)
    assert_parity(gpu, o64, o32, f"row staging, {walls}")


def test_reduce_is_exact_and_matches_oracle():
    """tslb_reduce (FP64 on the device) against numpy FP64 sums of the same
    downloaded state, and against the oracle's diagnostics at FP32 level."""
    from entropicthreadsafe_b200.solver import Lattice
    p, f = small_droplet()
    n = f["rho"].shape[0]
    with Lattice(p, n, n, n) as lat:
        lat.upload_moments(f)
        lat.step(20)
        st = lat.download()
        rg = lat.reduce()
    rho = st["rho"].astype(np.float64)
    phi = st["phi"].astype(np.float64)
    # rho is downloaded as 1 + (rho - 1) rounded to float, hence 1e-7 per node
    assert abs(rg["mass"] - rho.sum()) <= 1e-7 * rho.size
    assert abs(rg["mass_a"] - (rho * (1 + phi) / 2).sum()) <= 1e-7 * rho.size
    mom = (rho * st["u"]).sum()
    assert abs(rg["mom_x"] - mom) <= 1e-9 * rho.size
    _, ro = run_oracle(p, f, 20, fp64=True)
    for k, name in enumerate(capi.RED_NAMES):
        if name in ("mass", "mass_a", "mass_b", "rho_in", "rho_out", "n_in"):
            assert abs(rg[name] - ro[k]) <= 1e-5 * max(1.0, abs(ro[k])), name
        elif name in ("kinetic", "umax", "dp"):
            assert abs(rg[name] - ro[k]) <= 1e-2 * abs(ro[k]) + 1e-12, name


def test_reduce_is_deterministic():
    """The FP64 diagnostics add the per-block partials in block order: the
    same state gives bit-equal results on every call, also on a lattice large
    enough that every block of the reduction holds nodes."""
    from entropicthreadsafe_b200.solver import Lattice
    p, f = workloads.channel(nz=64, ndrops=10)
    nz, ny, nx = f["rho"].shape
    with Lattice(p, nx, ny, nz) as lat:
        lat.upload_moments(f)
        lat.step(3)
        runs = [lat.reduce() for _ in range(5)]
        st = lat.download()
    for r in runs[1:]:
        assert r == runs[0]
    rho = st["rho"].astype(np.float64)
    u2 = (st["u"].astype(np.float64) ** 2 + st["v"].astype(np.float64) ** 2 + st["w"].astype(np.float64) ** 2)
    assert abs(runs[0]["mass"] - rho.sum()) <= 1e-7 * rho.size
    assert abs(runs[0]["umax"] - np.sqrt(u2.max())) <= 1e-6 * np.sqrt(u2.max())


def test_uniform_colour_is_kept_exactly():
    """A single-colour flow (phi = -1 everywhere) keeps phi bit-exactly: the
    colour update is an increment that vanishes where phi is uniform."""
    p, f = workloads.channel(nx=40, ny=24, nz=20, ndrops=0, gx=2.5e-5)
    f["phi"][:] = -1.0
    gpu, _ = run_gpu(p, f, 50)
    assert np.all(gpu["phi"] == -1.0)


@pytest.mark.parametrize("walls", ["periodic", "bounceback_z", "moving_wall_z"])
def test_single_colour_kernel_matches_pinned_phase_field_oracle(walls):
    """The colour kernel with one colour everywhere, no force and equal
    relaxation times against the phase-field oracle at sigma = 0, whose f
    step is the reference's fused_TSLB_1c pinned by the golden vectors: the
    colour kernel's equilibrium, regularization, streaming and walls."""
    nx, ny, nz = 40, 12, 10
    bc = [capi.BC_PERIODIC] * 6
    bcu = [[0.0, 0.0, 0.0]] * 6
    if walls != "periodic":
        bc[capi.FACE_ZM] = capi.BC_BOUNCEBACK
        bc[capi.FACE_ZP] = capi.BC_BOUNCEBACK if walls == "bounceback_z" else capi.BC_VELOCITY
        if walls == "moving_wall_z":
            bcu = [[0.0, 0.0, 0.0]] * 5 + [[0.03, 0.0, 0.0]]
    rng = np.random.default_rng(7)
    f = workloads.empty_fields(nx, ny, nz)
    for k in ("u", "v", "w"):
        f[k][:] = rng.normal(0, 0.02, f[k].shape)
    for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        f[k][:] = rng.normal(0, 1e-4, f[k].shape)
    f["rho"][:] = 1.0 + rng.normal(0, 1e-3, f["rho"].shape)
    f["phi"][:] = 1.0
    pc = capi.make_params(mode=capi.MODE_COLOUR, tau_a=0.7, tau_b=0.7, sigma=0.01, beta=0.7, bc=bc, bc_u=bcu,
                          bc_phi=[1.0] * 6, wall_phi_mode=1)
    pp = capi.make_params(mode=capi.MODE_PHASEFIELD, tau_a=0.7, sigma=0.0, bc=bc, bc_u=bcu, bc_phi=[1.0] * 6)
    gpu, _ = run_gpu(pc, f, 40)
    o64, _ = run_oracle(pp, f, 40, fp64=True)
    o32, _ = run_oracle(pp, f, 40, fp64=False)
    assert np.all(gpu["phi"] == 1.0)
    for d in (gpu, o64, o32):
        d.pop("phi")
    eg = {k: rel_err(gpu[k], o64[k]) for k in gpu}
    e32 = {k: rel_err(o32[k], o64[k]) for k in gpu}
    bad = {k: (eg[k], e32[k]) for k in eg if eg[k] > max(TARGET, TOL_FACTOR * e32[k])}
    assert not bad, (walls, bad)


def test_colour_droplet_bounceback_all_faces():
    """Walls on x, y and z faces (lateral solid sources and solid planes)."""
    p, f = workloads.droplet(n=20, radius=5.0, tau=0.9, sigma=0.01, beta=0.7)
    for face in range(6):
        p.bc[face] = capi.BC_BOUNCEBACK
    p.wall_phi_mode = 1
    p.force[0], p.force[2] = 1e-5, -1e-5
    gpu, _ = run_gpu(p, f, 60)
    o64, _ = run_oracle(p, f, 60, fp64=True)
    o32, _ = run_oracle(p, f, 60, fp64=False)
    assert_parity(gpu, o64, o32, "colour box")


def degenerate_fields(dims, mode, seed):
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    f = workloads.empty_fields(nx, ny, nz)
    if mode == capi.MODE_COLOUR:
        f["phi"][:] = rng.uniform(-0.9, 0.9, f["phi"].shape)
    else:
        f["phi"][:] = rng.uniform(0.05, 0.95, f["phi"].shape)
    for k in ("u", "v", "w"):
        f[k][:] = rng.normal(0.0, 0.01, f[k].shape)
    f["rho"][:] = 1.0 + rng.normal(0.0, 1e-3, f["rho"].shape)
    return f


# On lattices one node thick some components of u and Pi^neq stay near zero
# (a single node relaxes to equilibrium: Pi^neq ~ 1e-17 in FP64), where
# max|a - b| / max|b| compares round-off with round-off.  These cases scale
# each component's error by the largest component of its tensor (u, v, w;
# the six Pi^neq), and Pi^neq at least by max |u|^2, the momentum flux rho uu
# it is the non-equilibrium remainder of (1e-6 for the others).
GROUPS = (("u", "v", "w"), ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"))


def grouped_errors(a, b):
    out = {}
    uu = float(max((np.asarray(b["u"], np.float64) ** 2 + np.asarray(b["v"], np.float64) ** 2 +
                    np.asarray(b["w"], np.float64) ** 2).max(), 1e-6))
    for ks in GROUPS:
        least = uu if ks[0] == "pxx" else 1e-6
        den = max(max(np.abs(np.asarray(b[k], np.float64)).max() for k in ks), least)
        for k in ks:
            out[k] = float(np.abs(np.asarray(a[k], np.float64) - b[k]).max() / den)
    d = np.asarray(b["rho"], np.float64) - 1.0
    out["rho-1"] = float(np.abs(np.asarray(a["rho"], np.float64) - 1.0 - d).max() / max(np.abs(d).max(), 1e-6))
    out["phi"] = float(np.abs(np.asarray(a["phi"], np.float64) - b["phi"]).max() / max(np.abs(b["phi"]).max(), 1e-6))
    return out


def assert_parity_grouped(gpu, o64, o32, label):
    eg, e32 = grouped_errors(gpu, o64), grouped_errors(o32, o64)
    print(label, {k: f"{v:.1e}" for k, v in eg.items()})
    bad = {k: (eg[k], e32[k]) for k in eg if eg[k] > max(TARGET, TOL_FACTOR * e32[k])}
    assert not bad, f"{label}: field: (gpu err, fp32 floor) {bad}"


@pytest.mark.parametrize("mode", [capi.MODE_COLOUR, capi.MODE_PHASEFIELD], ids=["colour", "phasefield"])
@pytest.mark.parametrize("dims", [(1, 1, 1), (1, 5, 7), (6, 1, 5), (5, 6, 1), (3, 2, 37), (4, 1, 6)],
                         ids=lambda d: "x".join(map(str, d)))
def test_degenerate_sizes(mode, dims):
    """Periodic lattices one node thick along one or more axes (and a single
    node): every neighbour along such an axis is the node itself, reached by
    the same modular wrap as the oracle's (mpi_module.f90:2083-2118)."""
    p, _ = workloads.droplet(n=8, radius=2.0, mode=mode)
    f = degenerate_fields(dims, mode, seed=sum(dims))
    gpu, _ = run_gpu(p, f, 20)
    o64, _ = run_oracle(p, f, 20, fp64=True)
    o32, _ = run_oracle(p, f, 20, fp64=False)
    assert_parity_grouped(gpu, o64, o32, f"degenerate {dims}")


def test_one_column_between_walls():
    """A 1 x 1 x 12 column between bounce-back walls (z), two colour layers and
    a body force along x: x and y are one node thick and periodic."""
    p, _ = workloads.droplet(n=8, radius=2.0)
    p.bc[capi.FACE_ZM] = p.bc[capi.FACE_ZP] = capi.BC_BOUNCEBACK
    p.wall_phi_mode = 1
    p.force[0] = 1e-5
    f = degenerate_fields((1, 1, 12), capi.MODE_COLOUR, seed=7)
    f["phi"][:] = -1.0
    f["phi"][:6] = 1.0
    gpu, _ = run_gpu(p, f, 60)
    o64, _ = run_oracle(p, f, 60, fp64=True)
    o32, _ = run_oracle(p, f, 60, fp64=False)
    assert_parity_grouped(gpu, o64, o32, "one column")


@pytest.mark.parametrize("mode", ["colour", "phasefield", "single"])
def test_periodic_shift_is_bit_exact(mode):
    """Translation invariance, bit for bit: on a fully periodic lattice,
    stepping a state shifted by (5, 3, 2) nodes gives the shifted result of
    stepping the state itself.  The shift moves every node to another place
    in the 32 x 8 tiles of the step: own nodes of a tile become rim nodes of
    its neighbours and rows move between the warps that compute the rim and
    those that do not, so this holds only if a node's coefficients are the
    same numbers wherever the step computes them."""
    nx, ny, nz = 64, 24, 16
    m = {"colour": capi.MODE_COLOUR, "phasefield": capi.MODE_PHASEFIELD, "single": capi.MODE_SINGLE}[mode]
    if m == capi.MODE_SINGLE:
        p = capi.make_params(mode=m, tau_a=0.6, force=[1e-5, 0.0, 0.0])
    elif m == capi.MODE_PHASEFIELD:
        p = capi.make_params(mode=m, tau_a=0.7, tau_b=0.7, sigma=0.01, sharp_c=0.9)
    else:
        p = capi.make_params(mode=m, tau_a=0.7, tau_b=0.9, sigma=0.01, beta=0.7, grad_threshold=1e-3,
                             force=[1e-5, 0.0, 0.0])
    rng = np.random.default_rng(11)
    f = workloads.empty_fields(nx, ny, nz)
    for k in ("u", "v", "w"):
        f[k][:] = rng.normal(0, 0.02, f[k].shape)
    for k in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        f[k][:] = rng.normal(0, 1e-4, f[k].shape)
    f["rho"][:] = 1.0 + rng.normal(0, 1e-3, f["rho"].shape)
    if m != capi.MODE_SINGLE:
        z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        r = np.sqrt((x - 20.3) ** 2 + (y - 9.6) ** 2 + (z - 7.2) ** 2)
        t = np.tanh((6.0 - r) / 2.0)
        f["phi"][:] = 0.5 * (1.0 + t) if m == capi.MODE_PHASEFIELD else t
    shift, axes = (2, 3, 5), (0, 1, 2)   # (z, y, x) of the (nz, ny, nx) arrays
    a, _ = run_gpu(p, f, 12)
    b, _ = run_gpu(p, {k: np.roll(v, shift, axes) for k, v in f.items()}, 12)
    for k in capi.FIELDS:
        ra = np.roll(np.asarray(a[k]), shift, axes)
        nbad = int(np.count_nonzero(ra != np.asarray(b[k])))
        assert nbad == 0, f"{mode}: field {k} differs at {nbad} nodes after the shift"
