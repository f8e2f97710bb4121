"""Regenerates tests/golden/golden_large.npz from the REFERENCE ITSELF, at the benchmark's sizes.

Run in a checkout where the reference tree is present and oracle/_ref/ref_harness_omp has been
built (`make -C oracle`).  Each graph comes from the library's seeded generators (the same
calls the benchmark and the GPU tests make); the compiled reference (oracle/ref_harness.cpp over
the unmodified ParButterfly headers) counts and peels it, and the results are stored either in
full (the 2^18-edge R-MAT sample of the benchmark workload) or as SHA-256 digests of the dense
little-endian int64 result plus a seeded sample of entries (the larger graphs).  The digest of
each graph's four CSR arrays is stored too, so a test can tell a generator change from a
counting error.

Records (the reference's flags in brackets):
  rmat18   : R-MAT 2^14 x 2^12, m = 2^18, (.55,.15,.15,.15), seed 2 — the benchmark workload's
             generator and flags at 1/64 of the edges [-rankType ACOCORE -per EDGE -countType HASH,
             wing peel -peelType BATCHS]: per-edge counts and wing numbers in full.
  rmat16   : R-MAT 2^16 x 2^14, m = 2^20, same parameters [-rankType ADEG -per VERT -countType
             BATCHS, tip peel BATCHS]: per-vertex counts and tip numbers (digests).
  plaw10m  : |U| = 1e6 power-law degrees (alpha 2, capped at |V| = 1e5), m = 1e7, seed 3 — the
             skewed Zipf-degree workload at 1/10 of its edges [ADEG, VERT, BATCHS, tip BATCHS]:
             per-vertex counts and tip numbers (digests).  Its largest count exceeds 2^32; the
             reference's 32-bit buckets still give the 64-bit answer on this graph (the C
             restatement, with 64-bit buckets, agrees).
  c2count  : the full benchmark graph, R-MAT 2^20 x 2^18, m = 2^24, seed 2 [ACOCORE, EDGE, HASH]:
             per-edge counts (digest) and the total.  Its wing peel does not finish within hours
             on the reference, so the reference's own wing numbers at this size are not recorded.
  c2wing   : (--c2-wing) wing numbers of the full benchmark graph from the C restatement's
             bucket-queue wing peel (oracle/pb_oracle_fast.c), run on per-edge counts whose
             digest equals the reference's c2count digest.  The restatement is pinned to the
             reference's own wing numbers on every golden graph and on rmat18; this record is
             the restatement's output, not the reference's (provenance stored with it).

  c3tip    : (--c3-tip) the skewed power-law-degree workload at full size (|U| = 1e6, |V| = 1e5,
             m = 1e8, seed 3): per-vertex counts and tip numbers (digests) from the C restatement
             (64-bit buckets; its counts exceed 2^32, where the reference's 32-bit buckets are not
             exact), pinned to the reference on plaw10m and every smaller fixture.

Usage: python tests/golden/make_golden_large.py [--skip-c2] [--c2-wing] [--c3-tip] [--threads N]
"""
import argparse
import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from parbutterfly_b200.graph import BipartiteGraph  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden_large.npz")
SAMPLE = 4096


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<i8").tobytes()).hexdigest()


def graph_digest(g) -> str:
    h = hashlib.sha256()
    h.update(np.array([g.nv, g.nu, g.m], dtype="<i8").tobytes())
    for a in (g.offsetsV, g.edgesV, g.offsetsU, g.edgesU):
        h.update(np.ascontiguousarray(a, dtype="<u4").tobytes())
    return h.hexdigest()


GRAPHS = {
    "rmat18": lambda: BipartiteGraph.rmat(14, 12, 1 << 18, 0.55, 0.15, 0.15, 0.15, 2),
    "rmat16": lambda: BipartiteGraph.rmat(16, 14, 1 << 20, 0.55, 0.15, 0.15, 0.15, 2),
    "plaw10m": lambda: BipartiteGraph.powerlaw_u(100_000, 1_000_000, 10_000_000, 2.0, 100_000, 3),
    "c2count": lambda: BipartiteGraph.rmat(20, 18, 1 << 24, 0.55, 0.15, 0.15, 0.15, 2),
}
FLAGS = {
    "rmat18": ("EDGE", "HASH", "ACOCORE", "BATCHS"),
    "rmat16": ("VERT", "BATCHS", "ADEG", "BATCHS"),
    "plaw10m": ("VERT", "BATCHS", "ADEG", "BATCHS"),
    "c2count": ("EDGE", "HASH", "ACOCORE", "NONE"),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-c2", action="store_true")
    ap.add_argument("--c2-wing", action="store_true", help="only add the c2wing record (needs c2count)")
    ap.add_argument("--c3-tip", action="store_true", help="only add the c3tip record")
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    a = ap.parse_args()
    if a.c2_wing:
        c2_wing(a.threads)
        return
    if a.c3_tip:
        c3_tip()
        return
    assert oracle.have_reference(), "build oracle/_ref first (make -C oracle)"
    out = {}
    if os.path.exists(OUT):
        with np.load(OUT) as z:
            out.update({k: z[k] for k in z.files})
    for name, make in GRAPHS.items():
        if a.skip_c2 and name == "c2count":
            continue
        g = make()
        per, ct, rank, peel = FLAGS[name]
        t0 = time.time()
        r = oracle.run_reference(g, per, ct, rank, peel, threads=a.threads)
        out[f"{name}/graph_sha"] = np.array(graph_digest(g))
        out[f"{name}/flags"] = np.array(" ".join(FLAGS[name]))
        out[f"{name}/use_v_wside_total"] = np.array([int(r["use_v"]), r["w_side"], r["total"]], dtype=np.int64)
        out[f"{name}/count_sha"] = np.array(digest(r["count"]))
        rng = np.random.default_rng(1234)
        idx = np.sort(rng.choice(r["count"].size, size=min(SAMPLE, r["count"].size), replace=False))
        out[f"{name}/sample_idx"] = idx.astype(np.int64)
        out[f"{name}/count_sample"] = r["count"][idx]
        if r["peel"] is not None:
            out[f"{name}/peel_sha"] = np.array(digest(r["peel"]))
            out[f"{name}/peel_sample"] = r["peel"][idx]
        if name == "rmat18":  # in full: the benchmark workload's small sample
            assert r["count"].max() < 2 ** 32 and r["peel"].max() < 2 ** 32
            out[f"{name}/count"] = r["count"].astype(np.uint32)
            out[f"{name}/peel"] = r["peel"].astype(np.uint32)
        print(f"{name}: nv={g.nv} nu={g.nu} m={g.m} total={r['total']} count_s={r['count_s']:.2f} "
              f"peel_s={r['peel_s']:.2f} wall={time.time() - t0:.1f}s", flush=True)
        np.savez_compressed(OUT, **out)


def c2_wing(threads):
    os.environ["OMP_NUM_THREADS"] = str(threads)
    with np.load(OUT) as z:
        out = {k: z[k] for k in z.files}
    g = GRAPHS["c2count"]()
    assert graph_digest(g) == str(out["c2count/graph_sha"])
    t0 = time.time()
    c, _ = oracle.count(g, "EDGE", "ACOCORE")
    assert digest(c) == str(out["c2count/count_sha"]), "oracle counts differ from the reference's"
    t1 = time.time()
    wing, rounds = oracle.peel_edge_fast(g, c)
    t2 = time.time()
    rng = np.random.default_rng(1234)
    idx = np.sort(rng.choice(wing.size, size=SAMPLE, replace=False))
    out["c2wing/graph_sha"] = out["c2count/graph_sha"]
    out["c2wing/provenance"] = np.array("oracle/pb_oracle_fast.c bucket-queue wing peel of the reference-matching "
                                        "per-edge counts (c2count digest)")
    out["c2wing/peel_sha"] = np.array(digest(wing))
    out["c2wing/sample_idx"] = idx.astype(np.int64)
    out["c2wing/peel_sample"] = wing[idx]
    out["c2wing/rounds_max"] = np.array([rounds, int(wing.max())], dtype=np.int64)
    np.savez_compressed(OUT, **out)
    print(f"c2wing: count {t1 - t0:.1f}s wing {t2 - t1:.1f}s rounds {rounds} max {int(wing.max())}", flush=True)


def c3_tip():
    g = BipartiteGraph.powerlaw_u(100_000, 1_000_000, 100_000_000, 2.0, 100_000, 3)
    t0 = time.time()
    c, w_rank = oracle.count(g, "VERT", "ADEG")
    t1 = time.time()
    tip, rounds = oracle.peel_vert(g, c)
    t2 = time.time()
    with np.load(OUT) as z:
        out = {k: z[k] for k in z.files}
    rng = np.random.default_rng(1234)
    idx = np.sort(rng.choice(c.size, size=SAMPLE, replace=False))
    out["c3tip/graph_sha"] = np.array(graph_digest(g))
    out["c3tip/provenance"] = np.array("oracle/pb_oracle.c ranked count (ADEG, VERT) and 64-bit-bucket tip peel")
    out["c3tip/count_sha"] = np.array(digest(c))
    out["c3tip/peel_sha"] = np.array(digest(tip))
    out["c3tip/sample_idx"] = idx.astype(np.int64)
    out["c3tip/count_sample"] = c[idx]
    out["c3tip/peel_sample"] = tip[idx]
    out["c3tip/total_rounds_wrank"] = np.array([int(c.sum()) // 2, rounds, w_rank], dtype=np.int64)
    np.savez_compressed(OUT, **out)
    print(f"c3tip: count {t1 - t0:.1f}s tip {t2 - t1:.1f}s rounds {rounds} total {int(c.sum()) // 2}", flush=True)


if __name__ == "__main__":
    main()
