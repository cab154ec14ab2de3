"""Multi-GPU sharding of independent units (batched BA windows): one process
per GPU, each optimizing its own windows with no communication on the data
path; only the timing (max over ranks) and the result summary cross ranks."""


def window_cost(cameras, points, mean_obs=4.4):
    """Estimated device work of one window: its edges (linearization, Schur
    pairs, chi2) plus the dense factorization of its reduced camera system."""
    n = 6 * cameras
    return points * mean_obs * 40.0 + n * n * n / 3.0


def assign_windows(costs, world):
    """Longest-processing-time assignment: windows by decreasing cost, each to
    the rank with the least total so far (ties to the lower rank). The same on
    every rank; every window on exactly one rank. Returns per rank the window
    indices in increasing order."""
    order = sorted(range(len(costs)), key=lambda w: (-costs[w], w))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for w in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(w)
        load[r] += costs[w]
    return [sorted(x) for x in out]
