"""Run the engine on a Vite file or a named synthetic graph and print one JSON
line of run statistics per run.

  python -m nido_b200 (--file graph.bin | --workload rmat22|rmat20|planted|sbm | --many NGRAPHS)
                      [--many-edges 1.5e9] [--runs 1] [-b 2] [-t 1e-6] [-i 500] [--tie nido] [--tune]
                      [--host-loop]

--many runs the batched engine (nido_batch_run) over the many-graph set of
NGRAPHS graphs (SBM / R-MAT mix, scaled to --many-edges directed edges).
"""
import argparse
import json

from . import capi, workloads


def main():
    ap = argparse.ArgumentParser(prog="python -m nido_b200")
    src = ap.add_mutually_exclusive_group(required=True)
    src.add_argument("--file")
    src.add_argument("--workload")
    src.add_argument("--many", type=int, metavar="NGRAPHS")
    ap.add_argument("--many-edges", type=float, default=1.5e9)
    ap.add_argument("--runs", type=int, default=1)
    ap.add_argument("-b", type=int, default=2)
    ap.add_argument("-t", type=float, default=1e-6)
    ap.add_argument("-i", type=int, default=500)
    ap.add_argument("--tie", choices=["smallest", "nido"], default="smallest")
    ap.add_argument("--tune", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--host-loop", action="store_true", help="drive the iteration loop from the host")
    a = ap.parse_args()
    tie = capi.NIDO_TIE_NIDO if a.tie == "nido" else capi.NIDO_TIE_SMALLEST_ID
    if a.many:
        vbase, U, _ = workloads.many_graphs_packed(a.many, 4, a.many_edges)
        with capi.Context(a.device) as ctx, capi.Batch(ctx, nbatches=a.b, packed=(vbase, U)) as B:
            for r in range(a.runs):
                _, q, ph, lo, st = B.run(tau=a.t, max_iter=a.i, tie=tie, tune=a.tune, host_loop=a.host_loop)
                print(json.dumps({"run": r, "ngraphs": len(vbase) - 1, "nv": U.nv, "ne": U.ne,
                                  "phases_max": int(ph.max()) if len(ph) else 0, "loops": st.total_loops,
                                  "total_ms": st.total_ms, "move_ms": st.move_ms, "q_ms": st.q_ms,
                                  "agg_ms": st.agg_ms,
                                  "move_gbs": st.move_bytes / (st.move_ms * 1e6) if st.move_ms else 0.0,
                                  "kernel_launches": st.kernel_launches,
                                  "host_ms": [round(x, 3) for x in st.host_ms]}), flush=True)
        return
    G = capi.read_vite(a.file) if a.file else workloads.single_graph(a.workload)
    with capi.Context(a.device) as ctx, capi.Graph(ctx, G, a.b) as g:
        for r in range(a.runs):
            _, st = g.run(tau=a.t, max_iter=a.i, tie=tie, tune=a.tune, host_loop=a.host_loop)
            print(json.dumps({"run": r, "nv": G.nv, "ne": G.ne, "phases": st.phases, "loops": st.total_loops,
                              "final_q": st.final_q, "total_ms": st.total_ms, "move_ms": st.move_ms,
                              "q_ms": st.q_ms, "agg_ms": st.agg_ms,
                              "move_gbs": st.move_bytes / (st.move_ms * 1e6) if st.move_ms else 0.0,
                              "kernel_launches": st.kernel_launches,
                              "tiers": g.tier_config().as_dict()}), flush=True)


if __name__ == "__main__":
    main()
