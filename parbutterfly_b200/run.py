"""Runs one named workload through the public API (used for profiling and ad-hoc timing).

    python -m parbutterfly_b200.run count-edge --graph rmat20    # pb_count_edge(HASH, ACOCORE)
    python -m parbutterfly_b200.run peel-edge --graph rmat15     # count, then pb_peel_edge
    python -m parbutterfly_b200.run peel-vert --graph rmat20     # count, then pb_peel_vert
    python -m parbutterfly_b200.run mlp-train                    # the cost model on the tensor cores
    python -m parbutterfly_b200.run batch-graph                  # the 256-graph batch as a CUDA graph

Graphs: rmat20 = bipartite R-MAT 2^20 x 2^18, m = 2^24, (.55,.15,.15,.15), seed 2 (the
benchmark workload); rmat15 = the same generator at 2^15 x 2^13, m = 2^19; rmat14 at
2^14 x 2^12, m = 2^18; c1 = uniform 4096 x 4096, m = 131072, seed 1; plaw10m / c3 = the
power-law-degree workload at 1e7 / 1e8 edges; generated on the device: c5 = bipartite R-MAT
2^26 x 2^24, m = 1e9, (.57,.19,.19,.05), seed 5, and rmat20d = the benchmark graph.
"""
import argparse
import sys

from . import butterflies as pb
from .graph import BipartiteGraph, workload

GRAPHS = {
    "rmat20": lambda: BipartiteGraph.rmat(20, 18, 1 << 24, 0.55, 0.15, 0.15, 0.15, 2),
    "rmat15": lambda: BipartiteGraph.rmat(15, 13, 1 << 19, 0.55, 0.15, 0.15, 0.15, 2),
    "rmat14": lambda: BipartiteGraph.rmat(14, 12, 1 << 18, 0.55, 0.15, 0.15, 0.15, 2),
    "plaw10m": lambda: BipartiteGraph.powerlaw_u(100_000, 1_000_000, 10_000_000, 2.0, 100_000, 3),
    "c3": lambda: workload("c3"),
    "c1": lambda: workload("c1"),
}


# Graphs generated on the device (pb_gen_rmat_device): the 1e9-edge R-MAT workload does not fit
# a host generator's memory.
DEVICE_GRAPHS = {
    "c5": lambda ctx: pb.gen_rmat_device(ctx, 26, 24, 1_000_000_000, 0.57, 0.19, 0.19, 0.05, 5),
    "rmat20d": lambda ctx: pb.gen_rmat_device(ctx, 20, 18, 1 << 24, 0.55, 0.15, 0.15, 0.15, 2),
}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["count-edge", "count-vert", "count-total", "peel-edge", "peel-vert", "mlp-train",
                                     "batch-graph", "batch-peel"])
    ap.add_argument("--graph", default="rmat15", choices=sorted(GRAPHS) + sorted(DEVICE_GRAPHS))
    ap.add_argument("--count-type", default="HASH")
    ap.add_argument("--rank-type", default="ACOCORE")
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--peel-parts", type=int, default=0, help="pb_opts.peel_parts of the peel calls")
    a = ap.parse_args(argv)
    if a.case == "mlp-train":
        import numpy as np
        rng = np.random.default_rng(0)
        X = rng.normal(size=(65536, 16)).astype(np.float32)
        y = (np.sin(X[:, 0]) + X[:, 1] * X[:, 2]).astype(np.float32)
        with pb.Context(0) as ctx:
            m = pb.SchedModel(ctx, seed=1)
            for _ in range(a.repeat):
                mse = m.train(m.COUNT, X, y, epochs=2, batch=8192, lr=3e-3)
                print(f"mlp-train rows={len(y)} mse={mse:.4f}")
            m.close()
        return 0
    if a.case == "batch-peel":
        gs = [BipartiteGraph.batch_member(k) for k in range(256)]
        with pb.Context(0) as ctx:
            dgs = [ctx.upload(g) for g in gs]
            cs = pb.count_batch(dgs, "BATCHS", "ADEG")
            print(f"batch-peel count ms={ctx.stats()['ms_count']:.1f}")
            for _ in range(a.repeat):
                pb.peel_batch(dgs, cs, peel_parts=a.peel_parts)
                s = ctx.stats()
                print(f"batch-peel ms={s['ms_peel']:.1f} rounds={s['peel_rounds']} parts={s['peel_parts']}")
            for dg in dgs:
                dg.close()
        return 0
    if a.case == "batch-graph":
        gs = [BipartiteGraph.batch_member(k) for k in range(256)]
        with pb.Context(0) as ctx:
            dgs = [ctx.upload(g) for g in gs]
            bg = pb.BatchGraph(dgs, "BATCHS", "ADEG", autotune=True)
            for _ in range(a.repeat):
                bg.run(copy_out=False)
                print(f"batch-graph replay ms={ctx.stats()['ms_count']:.1f}")
            bg.close()
        return 0
    with pb.Context(0) as ctx:
        if a.graph in DEVICE_GRAPHS:
            import time
            t0 = time.perf_counter()
            dg = DEVICE_GRAPHS[a.graph](ctx)
            print(f"generated on the device: nv={dg.nv} nu={dg.nu} m={dg.m} in {time.perf_counter() - t0:.1f} s")
        else:
            dg = ctx.upload(GRAPHS[a.graph]())
        for _ in range(a.repeat):
            if a.case in ("count-edge", "peel-edge"):
                e = pb.count_e(dg, a.count_type, a.rank_type)
                s = ctx.stats()
                print(f"count-edge w_rank={s['w_rank']} agg_ms={s['ms_agg_kernel']:.2f} total={int(e.sum()) // 4}")
                if a.case == "peel-edge":
                    pb.peel_e(dg, e, peel_parts=a.peel_parts)
                    s = ctx.stats()
                    print(f"peel-edge ms={s['ms_peel']:.1f} rounds={s['peel_rounds']} work={s['peel_work']} "
                          f"parts={s['peel_parts']} coarse_rounds={s['peel_coarse_rounds']} "
                          f"longest_part_rounds={s['peel_fine_rounds_max']}")
            elif a.case in ("count-vert", "peel-vert"):
                c = pb.count(dg, a.count_type, a.rank_type)
                s = ctx.stats()
                print(f"count-vert w_rank={s['w_rank']} agg_ms={s['ms_agg_kernel']:.2f} total={int(c.sum()) // 2}")
                if a.case == "peel-vert":
                    pb.peel(dg, c, peel_parts=a.peel_parts)
                    s = ctx.stats()
                    print(f"peel-vert ms={s['ms_peel']:.1f} rounds={s['peel_rounds']} work={s['peel_work']} "
                          f"parts={s['peel_parts']} coarse_rounds={s['peel_coarse_rounds']} "
                          f"longest_part_rounds={s['peel_fine_rounds_max']}")
            else:
                t = pb.count_total(dg, a.count_type, a.rank_type)
                s = ctx.stats()
                print(f"count-total w_rank={s['w_rank']} agg_ms={s['ms_agg_kernel']:.2f} total={t}")
        dg.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
