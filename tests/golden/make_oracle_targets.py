"""The FP64 oracle's trajectories on the full-size synthetic configurations,
written to tests/golden/oracle_targets.json.

Each entry holds the graph's digest (Graph.digest(): same digest, same
problem bit for bit), the solver, the iteration count and, per iteration,
the oracle's robust chi2 and number of LM trials. The full-size parity tests
check the GPU against the oracle run live and against these numbers; the
bench reads the final chi2 as the "FP64 chi2" its time-to-target is measured
against.

Configurations (the generators' defaults in g2o_b200/synth.py):
  ba    1000 VertexSE3Expmap / 200,000 VertexPointXYZ / ~1.03M EdgeProjectXYZ2UV,
        Huber, LM + Schur + block-Jacobi PCG, 20 iterations
  pg2d  3500 VertexSE2 / 5499 EdgeSE2, Gauss-Newton + Cholesky, 10 iterations
  pg3d  2500 VertexSE3 / 4759 EdgeSE3, LM + Cholesky, 20 iterations
  bal   356 VertexCameraBAL / 226,730 VertexPointBAL / ~1.27M EdgeObservationBAL,
        LM + Schur + block-Jacobi PCG (BlockSolver<9,3>), 10 iterations

Run from the repository root (a few minutes on 8 cores); names given on the
command line recompute only those entries and keep the others:
    python tests/golden/make_oracle_targets.py [ba pg2d pg3d bal]
"""
import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_targets.json")


def configs():
    from g2o_b200 import synth
    from g2o_b200.abi import ALGO_GAUSS_NEWTON, ALGO_LEVENBERG, LINEAR_CHOLESKY, LINEAR_PCG
    return {
        "ba": (synth.bundle_adjustment, dict(algorithm=ALGO_LEVENBERG, linear_solver=LINEAR_PCG), 20),
        "pg2d": (synth.pose_graph_2d, dict(algorithm=ALGO_GAUSS_NEWTON, linear_solver=LINEAR_CHOLESKY), 10),
        "pg3d": (synth.pose_graph_3d, dict(algorithm=ALGO_LEVENBERG, linear_solver=LINEAR_CHOLESKY), 20),
        "bal": (synth.bal_problem, dict(algorithm=ALGO_LEVENBERG, linear_solver=LINEAR_PCG), 10),
    }


def load():
    return json.load(open(OUT))


def main():
    from oracle import oracle
    oracle.build()
    names = sys.argv[1:] or list(configs())
    out = load() if sys.argv[1:] and os.path.exists(OUT) else {}
    for name, (make, prm, iters) in configs().items():
        if name not in names:
            continue
        g = make()
        t0 = time.perf_counter()
        o = oracle.OracleProblem(g, oracle.default_params(**prm), threads=os.cpu_count() or 1)
        done, st = o.optimize(iters)
        dt = time.perf_counter() - t0
        out[name] = {
            "digest": g.digest(), "poses": g.num_poses, "points": g.num_points, "edges": g.num_edges,
            "params": prm, "iterations": iters, "done": done,
            "chi2": [s["chi2"] for s in st], "levenberg_iterations": [s["levenberg_iterations"] for s in st],
            "final_chi2": st[-1]["chi2"],
        }
        print(f"{name}: {len(st)} iterations, final chi2 {st[-1]['chi2']:.12e}, {dt:.1f} s", flush=True)
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
