"""Generate golden vectors by evaluating the reference's own Fortran statements.

The reference (andreamontessori/entropicThreadsafe) is Fortran 90 + OpenACC
and no Fortran compiler exists in this container, so its step cannot be
built.  This script instead READS the reference source text, extracts the
statement blocks of the two-component phase-field step and evaluates each
statement unchanged with numpy, vectorised over all nodes of a small grid
(every loop body is free of loop-carried dependences, so the vectorised
evaluation equals the serial loop):

  initial conditions   recursive_2c_TSLB3D.f90:110-284
  moments pass         recursive_2c_TSLB3D.f90:351-539
  normals pass         recursive_2c_TSLB3D.f90:547-574
  collision + push     recursive_2c_TSLB3D.f90:612-832
  collision with force TSLB_2C-mpi/lb_kernels_module.f90:747-931
  bounce-back          boundary_cds_3D_module.f90:18-70 (at wall planes, and at
                       the nodes of an interior obstacle)
  moving walls         boundary_cds_3D_module.f90:413-571
  jet walls, inlet and boundary_cds_3D_module.f90:885-1050 (bcs_2c_turbulent_jet:
  outlet               bounce-back of the solid planes, regularized inlet at
                       k = 1, zero-gradient outlet at k = nz)
  single component     TSLB_2C-mpi/lb_kernels_module.f90:21-206 (moments_TSLB),
                       :423-566 (fused_TSLB_1c) and :583-730 (fused_TSLB_force_1c),
                       stepped as TSLB_2C-mpi/recursive_TSbcs_TSLB3.f90:285-353 does

Translation is mechanical: array references `a(i+1,j,k-1,q)` become
shifted numpy views, `x_db` literals drop the kind suffix, `if` blocks
become masks.  Periodic faces use the halo wrap of
TSLB_2C-mpi/mpi_module.f90:2083-2118 (populations) and of its scalar halo
exchange (phi, normals, moments), applied before and after the wall
conditions.  FP32 runs hold every variable in float32 (the reference's
db=4 build); FP64 runs hold every variable in float64.

The jet case stands a fixed inlet plane in for the host random_number
refresh of the inlet velocity (:866-877, compiler-defined): u = v = 0 and a
Gaussian w profile on the k = 1 plane, phi = 1 on a disc; the solid planes'
moments are never touched by the moments pass (it skips isfluid = 0 nodes),
so the plane stays as set, and the outlet plane's tangential velocity stays
at its initial 0.  The only rewrite of the source text: inside the
`elseif(k.eq.nz)` branch the index `nz-1` is the offset k-1.

Output: tests/golden/<case>.npz with the interior populations after the
initial conditions (the oracle's input) -- or, for the 32^3 case, the
FP32-representable initial moments (f = f^eq, so uploading them with
Pi^neq = 0 is the same state) --, the parameters, and the moment fields
after `nsteps` steps (the golden output; the 32^3 case keeps the FP64
result rounded to FP32 and the per-field spread of the FP32 run).  Run from
the repo root, with the reference checkout's path:

    python tests/golden/make_golden.py --reference <path to entropicThreadsafe>
"""
from __future__ import annotations

import argparse
import json
import os
import re

import numpy as np

ARRAYS = ("f", "g", "rho", "u", "v", "w", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz",
          "phi", "normx", "normy", "normz", "isfluid")
MOMENTS = ("rho", "u", "v", "w", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz", "phi")
REF_RE = re.compile(r"\b(" + "|".join(ARRAYS) + r")\s*\(([^()]*)\)")

BLOCKS = {
    "ic": ("recursive_2c_TSLB3D.f90", 110, 284),
    "moments": ("recursive_2c_TSLB3D.f90", 351, 539),
    "normals": ("recursive_2c_TSLB3D.f90", 547, 574),
    "collision": ("recursive_2c_TSLB3D.f90", 612, 832),
    "collision_force": ("TSLB_2C-mpi/lb_kernels_module.f90", 747, 931),
    "bounceback": ("boundary_cds_3D_module.f90", 18, 70),
    "couette": ("boundary_cds_3D_module.f90", 413, 571),
    "jet": ("boundary_cds_3D_module.f90", 885, 1050),
    # the single-component program (TSLB_2C-mpi/recursive_TSbcs_TSLB3.f90:285,346): moments_TSLB
    # and fused_TSLB_1c, and the module's forced collision fused_TSLB_force_1c
    "sc_moments": ("TSLB_2C-mpi/lb_kernels_module.f90", 21, 206),
    "sc_collision": ("TSLB_2C-mpi/lb_kernels_module.f90", 423, 566),
    "sc_collision_force": ("TSLB_2C-mpi/lb_kernels_module.f90", 583, 730),
}


# ---------------------------------------------------------------- parsing
def read_block(ref: str, fname: str, lo: int, hi: int) -> list[str]:
    with open(os.path.join(ref, fname)) as fh:
        lines = fh.read().split("\n")[lo - 1:hi]
    out, cur = [], ""
    for raw in lines:
        line = raw.split("!")[0].strip()  # drop comments (incl. !$acc)
        if not line:
            continue
        if line.endswith("&"):
            cur += line[:-1] + " "
            continue
        cur += line
        out.append(cur)
        cur = ""
    if cur:
        out.append(cur)
    return out


def parse(stmts: list[str]):
    """Return a tree: list of ('set', lhs, rhs) | ('if', [(cond, body), ...])."""
    root: list = []
    stack = [root]
    chains: list = []
    for s in stmts:
        low = s.replace(" ", "").lower()
        if low.startswith("if(") and low.endswith("then"):
            cond = s[s.index("(") + 1:s.rindex(")")]
            body: list = []
            node = ("if", [(cond, body)])
            stack[-1].append(node)
            chains.append(node)
            stack.append(body)
        elif low.startswith("elseif(") and low.endswith("then"):
            stack.pop()
            cond = s[s.index("(") + 1:s.rindex(")")]
            body = []
            chains[-1][1].append((cond, body))
            stack.append(body)
        elif low == "endif":
            stack.pop()
            chains.pop()
        else:
            lhs, rhs = s.split("=", 1)
            stack[-1].append(("set", lhs.strip(), rhs.strip()))
    assert len(stack) == 1, "unbalanced if/endif"
    return root


def _offset(arg: str, var: str) -> int:
    arg = arg.replace(" ", "")
    if arg == var:
        return 0
    if var == "k" and arg == "nz-1":
        # only inside the jet outlet branch `elseif(k.eq.nz)` (checked in run_case)
        return -1
    m = re.fullmatch(var + r"([+-]\d+)", arg)
    if not m:
        raise ValueError(f"unsupported index {arg!r}")
    return int(m.group(1))


def translate(expr: str) -> str:
    def ref(m):
        name, args = m.group(1), [a.strip() for a in m.group(2).split(",")]
        di, dj, dk = _offset(args[0], "i"), _offset(args[1], "j"), _offset(args[2], "k")
        q = args[3] if len(args) > 3 else "None"
        return f'_A("{name}",{di},{dj},{dk},{q})'

    e = REF_RE.sub(ref, expr)
    e = re.sub(r"(\d)_db\b", r"\1", e)
    return e


def translate_cond(cond: str) -> str:
    parts = re.split(r"\.and\.", cond, flags=re.I)
    out = []
    for p in parts:
        p = translate(p)
        p = re.sub(r"\.eq\.", "==", p, flags=re.I)
        p = re.sub(r"\.gt\.", ">", p, flags=re.I)
        p = re.sub(r"\.lt\.", "<", p, flags=re.I)
        p = re.sub(r"\bk\b", "_K", p)
        out.append("(" + p + ")")
    return " & ".join(out)


# -------------------------------------------------------------- execution
class Grid:
    def __init__(self, nx, ny, nz, dtype, periodic):
        self.n = (nx, ny, nz)
        self.dtype = dtype
        self.periodic = periodic  # per axis
        sh = (nx + 2, ny + 2, nz + 2)
        self.a = {name: np.zeros(sh, dtype) for name in ARRAYS if name not in ("f", "g", "isfluid")}
        self.a["f"] = np.zeros((27,) + sh, dtype)
        self.a["g"] = np.zeros((7,) + sh, dtype)
        self.a["isfluid"] = np.ones(sh, np.int32)
        self.K = np.arange(1, nz + 1).reshape(1, 1, nz)

    def view(self, name, di, dj, dk, q):
        nx, ny, nz = self.n
        arr = self.a[name] if q is None else self.a[name][q]
        return arr[1 + di:nx + 1 + di, 1 + dj:ny + 1 + dj, 1 + dk:nz + 1 + dk]

    def run(self, tree, consts: dict, mask=None):
        ns = dict(consts)
        ns["_A"] = self.view
        ns["_K"] = self.K
        ns["sqrt"] = np.sqrt
        ns["nz"] = self.n[2]
        if mask is None:
            mask = np.ones(self.n, bool)
        with np.errstate(all="ignore"):
            self._exec(tree, ns, mask)

    def _exec(self, tree, ns, mask):
        for node in tree:
            if node[0] == "set":
                _, lhs, rhs = node
                val = eval(translate(rhs), {"__builtins__": {}}, ns)
                m = REF_RE.fullmatch(lhs)
                if m:
                    tgt = eval(translate(lhs), {"__builtins__": {}}, ns)
                    tgt[...] = np.where(mask, val, tgt)
                else:
                    old = ns.get(lhs, np.zeros(self.n, self.dtype))
                    if not isinstance(old, np.ndarray) or old.shape != self.n:
                        old = np.zeros(self.n, self.dtype) + old
                    ns[lhs] = np.where(mask, val, old).astype(self.dtype)
            else:
                taken = np.zeros(self.n, bool)
                for cond, body in node[1]:
                    c = eval(translate_cond(cond), {"__builtins__": {}}, ns)
                    c = np.broadcast_to(c, self.n)
                    sub = mask & c & ~taken
                    taken |= c
                    self._exec(body, ns, sub)

    # periodic halo wraps ------------------------------------------------
    def wrap_scalar(self, name):
        arr = self.a[name]
        for ax in range(3):
            if not self.periodic[ax]:
                continue
            n = self.n[ax]
            lo = [slice(None)] * 3
            hi = [slice(None)] * 3
            src_lo = [slice(None)] * 3
            src_hi = [slice(None)] * 3
            lo[ax], src_lo[ax] = 0, n
            hi[ax], src_hi[ax] = n + 1, 1
            arr[tuple(lo)] = arr[tuple(src_lo)]
            arr[tuple(hi)] = arr[tuple(src_hi)]

    def wrap_pops(self):
        """Halo populations that left through a periodic face re-enter on the
        opposite side (intpbc: oi = mod(oi+nx-1,nx)+1), one axis at a time."""
        ex, ey, ez = CX, CY, CZ
        for name, cs in (("f", (ex, ey, ez)), ("g", (GXs, GYs, GZs))):
            arr = self.a[name]
            for ax in range(3):
                if not self.periodic[ax]:
                    continue
                n = self.n[ax]
                for q in range(arr.shape[0]):
                    c = cs[ax][q]
                    if c == 0:
                        continue
                    dst = [slice(None)] * 3
                    src = [slice(None)] * 3
                    if c < 0:
                        dst[ax], src[ax] = n, 0
                    else:
                        dst[ax], src[ax] = 1, n + 1
                    arr[q][tuple(dst)] = arr[q][tuple(src)]


CX = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, -1, 1, 1, -1]
CY = [0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, -1, 1, -1, 1]
CZ = [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1]
GXs = [0, 1, -1, 0, 0, 0, 0]
GYs = [0, 0, 0, 1, -1, 0, 0]
GZs = [0, 0, 0, 0, 0, 1, -1]


# ------------------------------------------------------------------ cases
CASES = {
    # fully periodic droplet, phase field, 2c collision block
    "pf_periodic": dict(n=(8, 8, 8), walls=None, collision="collision", nsteps=12,
                        tau=0.75, sigma=0.01, sharp_c=0.9, force=(0.0, 0.0, 0.0), uwall=0.0,
                        droplet=(4.5, 4.5, 4.5, 2.5), urand=0.01, seed=11),
    # x,y periodic, bounce-back z walls, body force (module collision block)
    "pf_walls_force": dict(n=(8, 6, 8), walls="bounceback", collision="collision_force", nsteps=12,
                           tau=0.8125, sigma=0.01, sharp_c=0.9, force=(2.0 ** -14, 0.0, 0.0),
                           uwall=0.0, droplet=(4.0, 3.5, 4.5, 1.8), urand=0.005, seed=12),
    # x,y periodic, regularized moving walls (Couette), single component (phi = 0)
    "couette": dict(n=(6, 6, 8), walls="couette", collision="collision", nsteps=12,
                    tau=0.625, sigma=0.0, sharp_c=0.9, force=(0.0, 0.0, 0.0), uwall=0.046875,
                    droplet=None, urand=0.005, seed=13),
    # x,y periodic, jet walls: fixed inlet plane at k = 1, zero-gradient outlet at k = nz
    "pf_jet": dict(n=(8, 8, 10), walls="jet", collision="collision", nsteps=12,
                   tau=0.75, sigma=0.01, sharp_c=0.9, force=(0.0, 0.0, 0.0), uwall=0.0,
                   droplet=None, urand=0.005, seed=14,
                   inlet=dict(centre=(4.5, 4.5), w=0.05, width=2.0, radius=2.5)),
    # fully periodic 32^3 droplet, 100 steps (initial moments stored, not populations)
    "pf_droplet32": dict(n=(32, 32, 32), walls=None, collision="collision", nsteps=100,
                         tau=0.8, sigma=0.01, sharp_c=0.9, force=(0.0, 0.0, 0.0), uwall=0.0,
                         droplet=(16.5, 16.5, 16.5, 8.0), urand=0.002, seed=15, moments_only=True),
    # fully periodic droplet beside an interior obstacle (isfluid = 0 nodes, i, j, k ranges
    # inclusive, 1-based): the bounce-back block acts at every solid node
    "pf_obstacle": dict(n=(8, 8, 8), walls=None, collision="collision", nsteps=12,
                        tau=0.75, sigma=0.01, sharp_c=0.9, force=(0.0, 0.0, 0.0), uwall=0.0,
                        droplet=(3.5, 4.5, 4.5, 2.0), urand=0.01, seed=18, obstacle=(5, 6, 3, 5, 3, 6)),
    # single component, fully periodic, from initial moments (random rho, u and Pi^neq)
    # (relaxation times that FP32 holds exactly, as the C-ABI's parameters are FP32)
    "sc_periodic": dict(n=(8, 6, 8), walls=None, single="sc_collision", nsteps=12, tau=0.6875,
                        force=(0.0, 0.0, 0.0), urand=0.02, pirand=1e-4, seed=16),
    "sc_force": dict(n=(8, 6, 8), walls=None, single="sc_collision_force", nsteps=12, tau=0.8125,
                     force=(2.0 ** -14, 2.0 ** -16, 0.0), urand=0.02, pirand=1e-4, seed=17),
}
# the moments of a single-component state (no phi)
SC_MOMENTS = MOMENTS[:-1]


def run_case_single(ref: str, cfg: dict, dtype):
    """The single-component program from a moment state: each step is the
    collision-and-push block, the periodic population exchange, and
    moments_TSLB (recursive_TSbcs_TSLB3.f90:285-353 in that order, entered
    after its moments pass).  The initial moments are FP32 numbers, the same
    for both precisions."""
    nx, ny, nz = cfg["n"]
    G = Grid(nx, ny, nz, dtype, (True, True, True))
    rng = np.random.default_rng(cfg["seed"])
    ic = {"rho": (1.0 + 1e-3 * rng.uniform(-1, 1, (nx, ny, nz))).astype(np.float32)}
    for name in ("u", "v", "w"):
        ic[name] = (cfg["urand"] * rng.uniform(-1, 1, (nx, ny, nz))).astype(np.float32)
    for name in ("pxx", "pxy", "pxz", "pyy", "pyz", "pzz"):
        ic[name] = (cfg["pirand"] * rng.uniform(-1, 1, (nx, ny, nz))).astype(np.float32)
    for name in SC_MOMENTS:
        G.a[name][1:-1, 1:-1, 1:-1] = ic[name].astype(dtype)
    t = dtype
    consts = {
        "p0": t(8.0) / t(27.0), "p1": t(2.0) / t(27.0), "p2": t(1.0) / t(54.0), "p3": t(1.0) / t(216.0),
        "omega": t(1.0) / t(cfg["tau"]),
        "fx": t(cfg["force"][0]), "fy": t(cfg["force"][1]), "fz": t(cfg["force"][2]),
    }
    moments = parse(read_block(ref, *BLOCKS["sc_moments"]))
    collision = parse(read_block(ref, *BLOCKS[cfg["single"]]))
    for _ in range(cfg["nsteps"]):
        G.run(collision, consts)
        G.wrap_pops()
        G.run(moments, consts)
    out = {name: G.a[name][1:nx + 1, 1:ny + 1, 1:nz + 1].copy() for name in SC_MOMENTS}
    return out, ic


def run_case(ref: str, cfg: dict, dtype):
    nx, ny, nz = cfg["n"]
    walls = cfg["walls"]
    periodic = (True, True, walls is None)
    G = Grid(nx, ny, nz, dtype, periodic)
    if walls:
        G.a["isfluid"][:, :, 1] = 0
        G.a["isfluid"][:, :, nz] = 0
    if cfg.get("obstacle"):
        i0, i1, j0, j1, k0, k1 = cfg["obstacle"]
        G.a["isfluid"][i0:i1 + 1, j0:j1 + 1, k0:k1 + 1] = 0
    rng = np.random.default_rng(cfg["seed"])
    i, j, k = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1), np.arange(1, nz + 1), indexing="ij")
    fluid = G.a["isfluid"][1:-1, 1:-1, 1:-1] == 1
    rho = 1.0 + 1e-3 * rng.uniform(-1, 1, (nx, ny, nz))
    uvw = cfg["urand"] * rng.uniform(-1, 1, (3, nx, ny, nz))
    phi = np.zeros((nx, ny, nz))
    if cfg["droplet"] is not None:
        cx, cy, cz, R = cfg["droplet"]
        r = np.sqrt((i - cx) ** 2 + (j - cy) ** 2 + (k - cz) ** 2)
        phi = 0.5 * (1 + np.tanh((R - r) / 1.0))
    ic = {}
    for name, val in (("rho", rho), ("u", uvw[0]), ("v", uvw[1]), ("w", uvw[2]), ("phi", phi)):
        G.a[name][1:-1, 1:-1, 1:-1] = np.where(fluid, val, 0.0).astype(dtype)
    inlet = None
    if walls == "jet":
        # the fixed inlet plane on the solid plane k = 1 (standing in for :866-877)
        spec = cfg["inlet"]
        ii, jj = np.meshgrid(np.arange(1, nx + 1), np.arange(1, ny + 1), indexing="ij")
        r2 = (ii - spec["centre"][0]) ** 2 + (jj - spec["centre"][1]) ** 2
        w_in = (spec["w"] * np.exp(-r2 / (2 * spec["width"] ** 2))).astype(np.float32)
        phi_in = (r2 <= spec["radius"] ** 2).astype(np.float32)
        G.a["u"][1:-1, 1:-1, 1] = 0
        G.a["v"][1:-1, 1:-1, 1] = 0
        G.a["w"][1:-1, 1:-1, 1] = w_in.astype(dtype)
        G.a["phi"][1:-1, 1:-1, 1] = phi_in.astype(dtype)
        inlet = np.stack([np.zeros_like(w_in), np.zeros_like(w_in), w_in, phi_in])   # (4, nx, ny)

    t = dtype
    consts = {
        "p0": t(8.0) / t(27.0), "p1": t(2.0) / t(27.0), "p2": t(1.0) / t(54.0), "p3": t(1.0) / t(216.0),
        "p0g": t(1.0) / t(4.0), "p1g": t(1.0) / t(8.0),
        "omega": t(1.0) / t(cfg["tau"]),
        "sigma": t(np.float32(cfg["sigma"])), "sharp_c": t(np.float32(cfg["sharp_c"])),
        "fx": t(cfg["force"][0]), "fy": t(cfg["force"][1]), "fz": t(cfg["force"][2]),
        "uwall": t(cfg["uwall"]),
    }
    tree = {name: parse(read_block(ref, *BLOCKS[name])) for name in BLOCKS if not name.startswith("sc_")}
    # the one rewritten index: `nz-1` of the jet block occurs in its k == nz branch only
    jet_text = " ".join(read_block(ref, *BLOCKS["jet"])).replace(" ", "")
    assert jet_text.count("nz-1") == 1 and jet_text.index("elseif(k.eq.nz)") < jet_text.index("nz-1")

    def run_block(name):
        # each block's outer `if(isfluid...)` is part of the tree
        G.run(tree[name], consts)

    run_block("ic")
    G.wrap_pops()
    kz = slice(2, nz) if walls else slice(1, nz + 1)
    f_in = G.a["f"][:, 1:nx + 1, 1:ny + 1, kz].copy()
    g_in = G.a["g"][:, 1:nx + 1, 1:ny + 1, kz].copy()

    moments_only = cfg.get("moments_only", False)
    if moments_only:
        # The state a step starts from is its moments.  The first moments pass
        # of the FP64 run (the initial populations, g written one node ahead)
        # rounded to FP32 is the stored initial state, and both runs start
        # from it instead of their own first moments pass.
        if dtype == np.float64:
            run_block("moments")
            for name in MOMENTS:
                ic[name] = G.a[name][1:nx + 1, 1:ny + 1, 1:nz + 1].astype(np.float32)
            run_case.ic64 = dict(ic)
        else:
            ic = dict(run_case.ic64)    # the FP64 run comes first (main)
        for name in MOMENTS:
            G.a[name][1:nx + 1, 1:ny + 1, 1:nz + 1] = ic[name].astype(dtype)
    for step in range(cfg["nsteps"]):
        if step > 0 or not moments_only:
            run_block("moments")
        G.wrap_scalar("phi")
        run_block("normals")
        for name in ("normx", "normy", "normz"):
            G.wrap_scalar(name)
        run_block(cfg["collision"])
        G.wrap_pops()
        if walls == "bounceback" or cfg.get("obstacle"):
            run_block("bounceback")
        elif walls == "couette":
            for name in MOMENTS:
                G.wrap_scalar(name)
            run_block("couette")
        elif walls == "jet":
            for name in MOMENTS:
                G.wrap_scalar(name)
            run_block("jet")
        G.wrap_pops()
    run_block("moments")
    out = {name: G.a[name][1:nx + 1, 1:ny + 1, kz].copy() for name in MOMENTS}
    return f_in, g_in, out, ic, inlet


def to_oracle_layout(a: np.ndarray) -> np.ndarray:
    """[..., i, j, k] (Fortran index order) -> [..., k, j, i] (x fastest, C order)."""
    return np.ascontiguousarray(np.swapaxes(a, -1, -3))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TSLB_REFERENCE"),
                    help="path of the reference checkout (or set TSLB_REFERENCE)")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--case", action="append", help="generate only these cases")
    args = ap.parse_args()
    if not args.reference:
        ap.error("give --reference (or TSLB_REFERENCE): the reference checkout to read the statements from")
    for name, cfg in CASES.items():
        if args.case and name not in args.case:
            continue
        if cfg.get("single"):
            res = {}
            outs = {}
            for tag, dt in (("fp64", np.float64), ("fp32", np.float32)):
                out, ic = run_case_single(args.reference, cfg, dt)
                outs[tag] = out
                for m in SC_MOMENTS:
                    res[f"{m}_{tag}"] = to_oracle_layout(out[m])
            for m in SC_MOMENTS:
                res[f"ic_{m}"] = to_oracle_layout(ic[m])
            meta = dict(cfg)
            meta["blocks"] = {k: list(BLOCKS[k]) for k in ("sc_moments", cfg["single"])}
            res["meta"] = np.array(json.dumps(meta))
            path = os.path.join(args.out, f"{name}.npz")
            np.savez_compressed(path, **res)
            d = max(np.abs(outs["fp32"][m] - outs["fp64"][m]).max() for m in SC_MOMENTS)
            print(f"{name}: wrote {path} ({os.path.getsize(path)} B); max |fp32-fp64| = {d:.3e}")
            continue
        res = {}
        outs = {}
        for tag, dt in (("fp64", np.float64), ("fp32", np.float32)):
            f_in, g_in, out, ic, inlet = run_case(args.reference, cfg, dt)
            outs[tag] = out
            if cfg.get("moments_only"):
                continue
            res[f"f_{tag}"] = to_oracle_layout(f_in)
            res[f"g_{tag}"] = to_oracle_layout(g_in)
            for m in MOMENTS:
                res[f"{m}_{tag}"] = to_oracle_layout(out[m])
        if cfg.get("moments_only"):
            for m in MOMENTS:
                res[f"ic_{m}"] = to_oracle_layout(ic[m])
            for m in MOMENTS:
                res[f"{m}_fp64"] = to_oracle_layout(outs["fp64"][m]).astype(np.float32)
            # spread of the reference's FP32 run, max|fp32 - fp64| / max|fp64| (rho as rho - 1)
            spread = {}
            for m in MOMENTS:
                a, b = outs["fp32"][m].astype(np.float64), outs["fp64"][m]
                if m == "rho":
                    a, b = a - 1.0, b - 1.0
                spread[m] = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))
            res["fp32_spread"] = np.array(json.dumps(spread))
        if inlet is not None:
            res["inlet"] = np.ascontiguousarray(np.swapaxes(inlet, -1, -2))   # (4, ny, nx): u, v, w, phi of the z- face
        meta = dict(cfg)
        meta["blocks"] = {k: list(v) for k, v in BLOCKS.items() if not k.startswith("sc_")}
        res["meta"] = np.array(json.dumps(meta))
        path = os.path.join(args.out, f"{name}.npz")
        np.savez_compressed(path, **res)
        d = max(np.abs(outs["fp32"][m] - outs["fp64"][m]).max() for m in MOMENTS)
        print(f"{name}: wrote {path} ({os.path.getsize(path)} B); max |fp32-fp64| = {d:.3e}")


if __name__ == "__main__":
    main()
