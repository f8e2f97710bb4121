"""Trains the learned scheduler's two cost models from traces the plain path logs.

Traces come from seeded synthetic training graphs that are disjoint from the benchmark
workloads (other seeds and sizes): bipartite R-MAT with three skews, Zipf-endpoint graphs and
uniform graphs.  With tracing in explore mode the plain path logs
  - count: one row per block-aggregator item of every count call (VERT and EDGE, HASH),
    with a random valid aggregation mode per item (target log2 SM cycles of the item);
  - peel:  one row per tip / wing peel call, sweeping the setting grid (tip: round batching of
    the two-phase schedule, grid-level thresholds, CTA count; wing: work units; target log2 ms of the
    call); larger graphs are traced for tip peeling only or wing peeling only, and batches of
    128 / 256 graphs (batch-generator members 1000+) for batch tip peeling.
Both MLPs are then trained on the GPU (tensor-core forward / backward, Adam) and saved.

    python -m parbutterfly_b200.sched_train --out sched.bin [--quick]
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import butterflies as pb
from .graph import BipartiteGraph

# (kind, args, seed): seeds 7000+ are used by no benchmark workload.
COUNT_GRAPHS = [
    ("rmat", (17, 15, 1 << 21, 0.55, 0.15, 0.15, 0.15), 7001),
    ("rmat", (18, 16, 1 << 22, 0.55, 0.15, 0.15, 0.15), 7002),
    ("rmat", (18, 17, 1 << 22, 0.57, 0.19, 0.19, 0.05), 7003),
    ("rmat", (16, 16, 1 << 21, 0.45, 0.25, 0.15, 0.15), 7004),
    ("zipf", (1 << 16, 1 << 14, 1 << 20, 1.5), 7005),
    ("zipf", (1 << 17, 1 << 15, 1 << 21, 1.2), 7006),
    ("uniform", (1 << 14, 1 << 13, 1 << 20), 7007),
]
PEEL_GRAPHS = [
    ("rmat", (15, 13, 1 << 18, 0.55, 0.15, 0.15, 0.15), 7101),
    ("rmat", (16, 14, 1 << 19, 0.55, 0.15, 0.15, 0.15), 7102),
    ("rmat", (16, 15, 1 << 19, 0.57, 0.19, 0.19, 0.05), 7103),
    ("zipf", (1 << 15, 1 << 13, 1 << 18, 1.5), 7104),
    ("uniform", (1 << 13, 1 << 12, 1 << 17), 7105),
    ("rmat", (17, 15, 1 << 21, 0.55, 0.15, 0.15, 0.15), 7106),
]
# Larger graphs traced for tip peeling only (a wing sweep of them would take minutes).
TIP_GRAPHS = [
    ("rmat", (19, 17, 1 << 23, 0.55, 0.15, 0.15, 0.15), 7201),
    ("rmat", (18, 17, 1 << 22, 0.57, 0.19, 0.19, 0.05), 7202),
]


def make(kind, args, seed) -> BipartiteGraph:
    if kind == "rmat":
        return BipartiteGraph.rmat(*args, seed)
    if kind == "zipf":
        return BipartiteGraph.zipf(*args, seed)
    return BipartiteGraph.uniform(*args, seed)


# Batches of graphs traced for tip peeling over every setting: members 1000+ of the batch
# generator (seeds 5000+; the benchmark batch uses members 0-255).
BATCH_SETS = [list(range(1000, 1128)), list(range(1200, 1456))]
# Larger graphs traced for wing peeling over every setting.
WING_GRAPHS = [
    ("rmat", (18, 16, 1 << 22, 0.55, 0.15, 0.15, 0.15), 7301),
    ("rmat", (19, 17, 1 << 23, 0.45, 0.25, 0.15, 0.15), 7302),
]


def collect(ctx: pb.Context, count_graphs=COUNT_GRAPHS, peel_graphs=PEEL_GRAPHS, peel_settings=48, log=print,
            tip_graphs=TIP_GRAPHS, wing_graphs=WING_GRAPHS, batch_sets=BATCH_SETS):
    """Explore-mode traces: returns (Xc, yc, Xp, yp)."""
    pb.trace_clear(ctx)
    pb.trace_set(ctx, "explore", seed=1)
    try:
        for spec in count_graphs:
            t0 = time.perf_counter()
            dg = ctx.upload(make(*spec))
            for rep in range(2):
                pb.count(dg, "HASH", "ADEG")
                pb.count_e(dg, "HASH", "ACOCORE")
            dg.close()
            log(f"[sched_train] count traces {spec[0]}{spec[1][:3]}: {time.perf_counter() - t0:.1f} s")
        for spec in peel_graphs:
            t0 = time.perf_counter()
            dg = ctx.upload(make(*spec))
            c = pb.count(dg, "BATCHS", "ADEG")
            ce = pb.count_e(dg, "BATCHS", "ADEG")
            for k in range(peel_settings):
                pb.peel(dg, c)
                pb.peel_e(dg, ce)
            dg.close()
            log(f"[sched_train] peel traces {spec[0]}{spec[1][:3]}: {time.perf_counter() - t0:.1f} s")
        for spec in tip_graphs:
            t0 = time.perf_counter()
            dg = ctx.upload(make(*spec))
            c = pb.count(dg, "BATCHS", "ADEG")
            for k in range(peel_settings):
                pb.peel(dg, c)
            dg.close()
            log(f"[sched_train] tip traces {spec[0]}{spec[1][:3]}: {time.perf_counter() - t0:.1f} s")
        for spec in wing_graphs:
            t0 = time.perf_counter()
            dg = ctx.upload(make(*spec))
            ce = pb.count_e(dg, "BATCHS", "ADEG")
            for c in range(3):  # every wing candidate (the sweep position of the next peel call)
                pb.trace_set(ctx, "explore", seed=c)
                pb.peel_e(dg, ce)
            dg.close()
            log(f"[sched_train] wing traces {spec[0]}{spec[1][:3]}: {time.perf_counter() - t0:.1f} s")
        for members in batch_sets:
            t0 = time.perf_counter()
            dgs = [ctx.upload(BipartiteGraph.batch_member(k)) for k in members]
            cs = pb.count_batch(dgs, "BATCHS", "ADEG")
            for c in range(48):  # every tip candidate
                pb.trace_set(ctx, "explore", seed=c)
                pb.peel_batch(dgs, cs)
            for dg in dgs:
                dg.close()
            log(f"[sched_train] batch tip traces {len(members)} graphs: {time.perf_counter() - t0:.1f} s")
    finally:
        pb.trace_set(ctx, "off")
    Xc, yc = pb.trace_rows(ctx, pb.SchedModel.COUNT)
    Xp, yp = pb.trace_rows(ctx, pb.SchedModel.PEEL)
    pb.trace_clear(ctx)
    return Xc, yc, Xp, yp


def train(ctx: pb.Context, Xc, yc, Xp, yp, seed=1, log=print) -> pb.SchedModel:
    m = pb.SchedModel(ctx, seed=seed)
    t0 = time.perf_counter()
    mse_c = m.train(m.COUNT, Xc, yc, epochs=40, batch=1024, lr=3e-3)
    mse_p = m.train(m.PEEL, Xp, yp, epochs=300, batch=64, lr=3e-3)
    log(f"[sched_train] trained on {len(yc)} count rows (mse {mse_c:.3f}) and {len(yp)} peel rows "
        f"(mse {mse_p:.3f}) in {time.perf_counter() - t0:.1f} s")
    return m


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--quick", action="store_true", help="fewer graphs and peel settings")
    a = ap.parse_args()
    ctx = pb.Context(a.device)
    cg, pg, ps, tg, wg, bs = COUNT_GRAPHS, PEEL_GRAPHS, 48, TIP_GRAPHS, WING_GRAPHS, BATCH_SETS
    if a.quick:
        cg, pg, ps, tg, wg, bs = COUNT_GRAPHS[::2], PEEL_GRAPHS[:2], 16, [], [], []
    Xc, yc, Xp, yp = collect(ctx, cg, pg, ps, tip_graphs=tg, wing_graphs=wg, batch_sets=bs)
    m = train(ctx, Xc, yc, Xp, yp)
    m.save(a.out)
    print(f"[sched_train] saved {a.out}")


if __name__ == "__main__":
    main()
