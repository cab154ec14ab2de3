"""Command-line runner, the counterpart of g2o_cli's `-solver <name> -i <n>`
(g2o/apps/g2o_cli/g2o.cpp:133-187) for the synthetic configurations:

    python -m g2o_b200.cli --config ba --solver lm_cuda_pcg6_3 -i 20 [-stats]
    python -m g2o_b200.cli --config windows --windows 64 --solver lm_cuda_mixed_fast -i 10
    python -m g2o_b200.cli --bal problem.txt --solver lm_cuda_pcg9_3 -i 5 -o out.txt
    python -m g2o_b200.cli --input graph.g2o -o graph_opt.g2o --solver lm_cuda -i 20

(g2o_b200/g2o_cuda_cli is the native counterpart for .g2o files, with g2o_cli's
options.)

Prints one line per iteration with chi2, lambda, trial and PCG counts and the
phase times (the fields of G2OBatchStatistics); for the batched windows, one
line per window with its iterations, trials and chi2.
"""
import argparse
import sys

from . import backend, synth

CONFIGS = {
    "ba": lambda: synth.bundle_adjustment(),
    "ba_small": lambda: synth.bundle_adjustment(num_cameras=100, num_points=20000, seed=99),
    "pg2d": lambda: synth.pose_graph_2d(),
    "pg3d": lambda: synth.pose_graph_3d(),
    "bal": lambda: synth.bal_problem(),
    "bal_small": lambda: synth.bal_problem(num_cameras=60, num_points=8000, seed=98),
    "windows": None,  # batched local BA windows (synth.windows), see run_windows
}


def run_windows(a, params):
    ws = synth.windows(which=list(range(min(max(a.windows, 1), 512))))
    cw = backend.CudaWindows(ws, params, device=a.device)
    cw.set_kernel_timing(a.stats)
    st = cw.optimize(a.iterations)
    print(f"# {len(ws)} windows, {sum(w.num_edges for w in ws)} edges; {st[0]['rounds']} LM rounds")
    for w, s in enumerate(st):
        print(f"window= {w}\t iterations= {s['iterations']}\t trials= {s['trials']}\t chi2_initial= "
              f"{s['chi2_initial']:.6f}\t chi2= {s['chi2']:.6f}\t choleskyThreads= {s['cholesky_threads']}")
    if a.stats:
        total, ks = cw.kernel_stats()
        print(f"# kernel launches: {total}")
        for k, (n, ms) in sorted(ks.items(), key=lambda kv: -kv[1][1]):
            print(f"#   {k:20s} {n:7d} {ms:10.3f} ms")
    cw.close()
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--config", default="ba", choices=sorted(CONFIGS))
    ap.add_argument("--solver", default="lm_cuda_pcg6_3")
    ap.add_argument("-i", "--iterations", type=int, default=20)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("-stats", "--stats", action="store_true", help="print per-kernel launch counts and times")
    ap.add_argument("--listSolvers", action="store_true")
    ap.add_argument("--windows", type=int, default=512, help="windows: how many of the 512 local BA windows")
    ap.add_argument("--input", help="a .g2o file to optimize instead of a synthetic configuration")
    ap.add_argument("-o", "--output", help="with --input / --bal: write the optimized graph here")
    ap.add_argument("--bal", help="a BAL problem file (the input of g2o's bal_example) to optimize, e.g. with "
                                  "--solver lm_cuda_pcg9_3")
    a = ap.parse_args(argv)
    fac = backend.OptimizationAlgorithmFactory.instance()
    if a.listSolvers:
        print("\n".join(fac.list_solvers()))
        return 0
    params = fac.construct(a.solver)
    if params is None:
        print(f"unknown solver {a.solver}", file=sys.stderr)
        return 1
    if a.config == "windows":
        return run_windows(a, params)
    gfile = None
    if a.bal:
        from .bal import read_bal
        g = read_bal(a.bal)
    elif a.input:
        from .g2ofile import G2oFile
        gfile = G2oFile.load(a.input)
        gid = gfile.fix_gauge()
        print(f"# {a.input}: {gfile.info()['num_vertices']} vertices, {gfile.info()['num_edges']} edges"
              + (f"; gauge fixed at vertex {gid}" if gid >= 0 else ""))
        g = gfile.graph()
        g.name = a.input
    else:
        g = CONFIGS[a.config]()
    prob = backend.CudaProblem(g, params, device=a.device)
    prob.set_kernel_timing(a.stats)
    chi0, rchi0 = prob.chi2()
    print(f"# {g.name}: {g.num_poses} poses, {g.num_points} points, {g.num_edges} edges; initial chi2 {rchi0:.6f}")
    done, stats = prob.optimize(a.iterations)
    for s in stats:
        print(f"iteration= {s['iteration']}\t chi2= {s['chi2']:.6f}\t lambda= {s['lambda']:.6e}\t "
              f"levenbergIter= {s['levenberg_iterations']}\t pcgIter= {s['iterations_linear_solver']}\t "
              f"time= {s['time_iteration']:.6f}")
    if a.stats:
        total, ks = prob.kernel_stats()
        print(f"# kernel launches: {total}")
        for k, (n, ms) in sorted(ks.items(), key=lambda kv: -kv[1][1]):
            print(f"#   {k:20s} {n:7d} {ms:10.3f} ms")
    if a.bal and a.output:
        from .bal import write_bal
        out = g.copy()
        out.pose_estimate, out.point_estimate = prob.estimates()
        write_bal(out, a.output)
    if gfile is not None and a.output:
        pose, point = prob.estimates()
        gfile.set_estimates(pose, point)
        gfile.save(a.output)
    prob.close()
    return 0 if done > 0 else 2


if __name__ == "__main__":
    sys.exit(main())
