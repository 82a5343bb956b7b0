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
  bounce-back          boundary_cds_3D_module.f90:18-70
  moving walls         boundary_cds_3D_module.f90:413-571

Translation is mechanical: array references `a(i+1,j,k-1,q)` become
shifted numpy views, `x_db` literals drop the kind suffix, `if` blocks
become masks.  Periodic faces use the halo wrap of
TSLB_2C-mpi/mpi_module.f90:2083-2118 (populations) and of its scalar halo
exchange (phi, normals, moments), applied before and after the wall
conditions.  FP32 runs hold every variable in float32 (the reference's
db=4 build); FP64 runs hold every variable in float64.

Output: tests/golden/<case>.npz with the interior populations after the
initial conditions (the oracle's input), the parameters, and the moment
fields after `nsteps` steps (the golden output).  Run from the repo root:

    python tests/golden/make_golden.py [--reference /root/reference]
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
}


def run_case(ref: str, cfg: dict, dtype):
    nx, ny, nz = cfg["n"]
    walls = cfg["walls"]
    periodic = (True, True, walls is None)
    G = Grid(nx, ny, nz, dtype, periodic)
    if walls:
        G.a["isfluid"][:, :, 1] = 0
        G.a["isfluid"][:, :, nz] = 0
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
    for name, val in (("rho", rho), ("u", uvw[0]), ("v", uvw[1]), ("w", uvw[2]), ("phi", phi)):
        G.a[name][1:-1, 1:-1, 1:-1] = np.where(fluid, val, 0.0).astype(dtype)

    t = dtype
    consts = {
        "p0": t(8.0) / t(27.0), "p1": t(2.0) / t(27.0), "p2": t(1.0) / t(54.0), "p3": t(1.0) / t(216.0),
        "p0g": t(1.0) / t(4.0), "p1g": t(1.0) / t(8.0),
        "omega": t(1.0) / t(cfg["tau"]),
        "sigma": t(np.float32(cfg["sigma"])), "sharp_c": t(np.float32(cfg["sharp_c"])),
        "fx": t(cfg["force"][0]), "fy": t(cfg["force"][1]), "fz": t(cfg["force"][2]),
        "uwall": t(cfg["uwall"]),
    }
    tree = {name: parse(read_block(ref, *BLOCKS[name])) for name in BLOCKS}

    def run_block(name):
        # each block's outer `if(isfluid...)` is part of the tree
        G.run(tree[name], consts)

    run_block("ic")
    G.wrap_pops()
    kz = slice(2, nz) if walls else slice(1, nz + 1)
    f_in = G.a["f"][:, 1:nx + 1, 1:ny + 1, kz].copy()
    g_in = G.a["g"][:, 1:nx + 1, 1:ny + 1, kz].copy()

    for _ in range(cfg["nsteps"]):
        run_block("moments")
        G.wrap_scalar("phi")
        run_block("normals")
        for name in ("normx", "normy", "normz"):
            G.wrap_scalar(name)
        run_block(cfg["collision"])
        G.wrap_pops()
        if walls == "bounceback":
            run_block("bounceback")
        elif walls == "couette":
            for name in MOMENTS:
                G.wrap_scalar(name)
            run_block("couette")
        G.wrap_pops()
    run_block("moments")
    out = {name: G.a[name][1:nx + 1, 1:ny + 1, kz].copy() for name in MOMENTS}
    return f_in, g_in, out


def to_oracle_layout(a: np.ndarray) -> np.ndarray:
    """[..., i, j, k] (Fortran index order) -> [..., k, j, i] (x fastest, C order)."""
    return np.ascontiguousarray(np.swapaxes(a, -1, -3))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    args = ap.parse_args()
    for name, cfg in CASES.items():
        res = {}
        for tag, dt in (("fp64", np.float64), ("fp32", np.float32)):
            f_in, g_in, out = run_case(args.reference, cfg, dt)
            res[f"f_{tag}"] = to_oracle_layout(f_in)
            res[f"g_{tag}"] = to_oracle_layout(g_in)
            for m in MOMENTS:
                res[f"{m}_{tag}"] = to_oracle_layout(out[m])
        meta = dict(cfg)
        meta["blocks"] = {k: list(v) for k, v in BLOCKS.items()}
        res["meta"] = np.array(json.dumps(meta))
        path = os.path.join(args.out, f"{name}.npz")
        np.savez_compressed(path, **res)
        d = max(np.abs(res[f"{m}_fp32"] - res[f"{m}_fp64"]).max() for m in MOMENTS)
        print(f"{name}: wrote {path} ({os.path.getsize(path)} B); max |fp32-fp64| = {d:.3e}")


if __name__ == "__main__":
    main()
