"""Launch-shape tuner of the GAMG V-cycle.

The knob it tunes is where the V-cycle switches from per-level launches (a few kernels per level,
each spread over the whole GPU) to the coarse tail (all remaining levels of a system in one launch
on a thread-block cluster, steps separated by the cluster barrier), and how wide that cluster is:

* cluster   - CTAs per system in the tail launch: 1, 2, 4 or 8 (1024 threads each);
* max_rows  - levels of at most this many rows go to the tail;
* full_rows - systems of at most this many level-0 rows run their whole V-cycle in the tail.

None of them changes a result: the tail performs the same row operations in the same order.  For a
mesh, every configuration that splits its levels differently is timed with CUDA events on full
GAMG-PCG solves (the production path: one graph launch per solve), and the fastest is kept.  The
results go to a per-device table (voluma_b200/tuning/<device>.json, one entry per mesh-size class:
level-0 rows and number of systems), which Mesh registration applies to every new mesh of the same
device (Mesh._apply_tuning: nearest size class, same single/batched kind).

    python -m voluma_b200.tune [--out voluma_b200/tuning] [--cases tgv128,tgv64,...]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE_DIR = os.path.join(HERE, "tuning")
_tables: dict = {}


def _slug(name: str) -> str:
    return "".join(ch if ch.isalnum() else "_" for ch in name).strip("_").lower()


def table_path(device_name: str, directory: str = TABLE_DIR) -> str:
    return os.path.join(directory, _slug(device_name) + ".json")


def load_table(device_name: str) -> list:
    if device_name not in _tables:
        p = os.environ.get("VLM_TUNING_TABLE") or table_path(device_name)
        try:
            with open(p) as f:
                t = json.load(f)
            _tables[device_name] = t.get("entries", []) if t.get("device") == device_name else []
        except (OSError, ValueError):
            _tables[device_name] = []
    return _tables[device_name]


def lookup(entries: list, rows0: int, nsys: int):
    """The entry of the nearest size class (log2 of the level-0 rows per system) of the same kind
    (one system or a batch); None when the table has none of that kind."""
    kind = [e for e in entries if (e["nsys"] > 1) == (nsys > 1)]
    if not kind:
        return None
    per = max(1, rows0 // max(1, nsys))
    return min(kind, key=lambda e: abs(math.log2(max(1, e["rows0"] // max(1, e["nsys"]))) - math.log2(per)))


def apply(mesh) -> dict | None:
    """Sets the tuned tail configuration of `mesh` (a voluma_b200.Mesh) from its device's table."""
    entries = load_table(mesh.ctx.device_name())
    e = lookup(entries, int(mesh.n_cells), int(getattr(mesh, "n_systems", 1)))
    if e is None:
        return None
    mesh.set_tail(e["cluster"], e["max_rows"], e["full_rows"])
    return e


# ------------------------------------------------------------------------------ measurement
def candidates(level_rows: list, clusters=(1, 2, 4, 8), max_per_thread: int = 4):
    """Configurations that split one system's levels differently: for each cluster size, the tail
    starting at level 0 (whole V-cycle) or at each coarse level whose rows the cluster covers with at
    most `max_per_thread` rows per thread."""
    out = []
    n0 = level_rows[0]
    padded = [(n + 31) // 32 * 32 for n in level_rows]  # coarse levels: rows padded to whole warps
    for cl in clusters:
        cap = 1024 * cl * max_per_thread
        if len(level_rows) > 1 and n0 <= cap:
            out.append((cl, 1, 2 * n0 + 64))  # the whole V-cycle in the tail (level 0 with its padding)
        for k in range(1, len(level_rows)):
            if padded[k] <= cap:
                out.append((cl, padded[k], 1))
    return out


def time_solves(mesh, d, up, b, ctrl, reps: int):
    """Median ms of `reps` device solves (CUDA events on the mesh's stream), the solution and the
    iteration count."""
    import torch
    import voluma_b200 as vb
    dev = torch.device("cuda", 0)
    st = torch.cuda.ExternalStream(mesh.ctx.stream(), device=dev)
    dd, du, db = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (d, up, b))
    x = torch.zeros(len(b), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    def one():
        with torch.cuda.stream(st):
            x.zero_()
        return vb.solve_ldu_device(mesh, dd.data_ptr(), du.data_ptr(), 0, db.data_ptr(), x.data_ptr(), ctrl)
    one()
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        perf = one()
        e1.record(st)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.median(ms)), x.cpu().numpy(), perf.iterations


def tune_system(mesh, d, up, b, ctrl, reps: int = 5, log=print) -> dict:
    """Times every distinct tail configuration of a single-system mesh; keeps the fastest on the mesh
    and returns its table entry."""
    sizes = [int(L["n"]) for L in mesh.gamg_levels()]
    default = mesh.tail_config()
    base, x0, it0 = time_solves(mesh, d, up, b, ctrl, reps)
    best = (base, default)
    log(f"  default {default}: {base:.3f} ms, {it0} iterations")
    for cfg in candidates(sizes):
        mesh.set_tail(*cfg)
        t, x, it = time_solves(mesh, d, up, b, ctrl, reps)
        # a launch configuration must not change a result: anything else is a defect, never a candidate
        same = it == it0 and np.array_equal(x, x0)
        log(f"  {cfg}: {t:.3f} ms{'' if same else '  RESULT DIFFERS - rejected'}")
        if same and t < best[0]:
            best = (t, cfg)
        if not same:
            raise RuntimeError(f"tail configuration {cfg} changed the solution ({it} vs {it0} iterations)")
    mesh.set_tail(*best[1])
    return {"rows0": sizes[0], "nsys": 1, "cluster": int(best[1][0]), "max_rows": int(best[1][1]),
            "full_rows": int(best[1][2]), "ms": best[0], "default_ms": base, "levels": sizes}


def _poisson_case(name):
    from voluma_b200 import mesh as vm
    if name.startswith("tgv"):
        n = int(name[3:])
        m = vm.box_mesh((n, n, n), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
    elif name.startswith("cavity"):
        n = int(name[6:])
        m = vm.box_mesh((n, n, 1), hi=(1.0, 1.0, 0.1), two_d=True)
    elif name.startswith("box"):
        n = int(name[3:])
        m = vm.box_mesh((n, n, n))
    else:
        raise ValueError(name)
    d, up = vm.poisson_matrix(m)
    rng = np.random.default_rng(20261203)
    b = rng.standard_normal(m["n_cells"])
    b -= b.mean()
    return m, d, up, b


def main():
    import voluma_b200 as vb
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TABLE_DIR)
    ap.add_argument("--cases", default="tgv128,tgv96,tgv64,box48,box32,cavity256,cavity128,cavity64")
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--precision", default="mixed")
    args = ap.parse_args()
    os.environ["VLM_TUNE"] = "0"  # tune from the built-in defaults
    ctx = vb.default_context()
    name = ctx.device_name()
    entries = []
    for case in args.cases.split(","):
        m, d, up, b = _poisson_case(case)
        mesh = vb.Mesh.from_arrays(m)
        ctrl = vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 1000, precision=args.precision)
        t0 = time.time()
        print(f"{case}: {m['n_cells']} cells", flush=True)
        e = tune_system(mesh, d, up, b, ctrl, args.reps)
        e["case"] = case
        print(f"  -> {e['cluster']}, {e['max_rows']}, {e['full_rows']}: {e['ms']:.3f} ms "
              f"(default {e['default_ms']:.3f}); {time.time() - t0:.0f} s", flush=True)
        entries.append(e)
        mesh.close()
    os.makedirs(args.out, exist_ok=True)
    out = table_path(name, args.out)
    with open(out, "w") as f:
        json.dump({"device": name, "how": "voluma_b200.tune: median of %d GAMG-PCG solves (%s precision) per "
                                          "configuration, CUDA events" % (args.reps, args.precision),
                   "entries": entries}, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
