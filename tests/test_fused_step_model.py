"""The argument behind k_sweep_changed, checked on a host model.

k_sweep_changed runs a plain iteration after a dense changed set U without
materialising the frontier: row v is active iff an in-edge comes from U, and
only the in-edges from U are folded.  That is exact because of an invariant of
the plain loop: after every iteration, each edge u -> v either has its source
in the iteration's changed set or already satisfies V[v] <= comp(V[u]) (when u
last changed, v was activated and pulled it).  This test runs a synchronous
(Jacobi) model of the plain loop -- every active row folds every in-edge --
next to the same loop whose pull folds only the in-edges from the previous
changed set, on the config-1 graph and on random graphs, and requires the same
values, active rows and traversed edges in every iteration."""
import numpy as np
import pytest

from oracle import oracle as O

INF = np.uint64(0xFFFFFFFF)


def comp(vals, w):
    s = vals.astype(np.uint64) + w.astype(np.uint64)
    return np.where((vals.astype(np.uint64) == INF) | (s > INF), INF, s)


def plain_loop(R, C, E, V0, source, fused):
    """Per iteration: (values, active rows, edges of active rows)."""
    n = V0.shape[0]
    V = V0.astype(np.uint64)
    row = np.repeat(np.arange(n), np.diff(R.astype(np.int64)))
    U = np.zeros(n, bool)
    U[source] = True
    out = []
    for _ in range(4 * n + 8):
        from_changed = U[C]
        active = np.zeros(n, bool)
        active[row[from_changed]] = True
        if not active.any():
            break
        use = (active[row] & (from_changed if fused else True))
        cand = np.full(n, INF, np.uint64)
        np.minimum.at(cand, row[use], comp(V[C[use]], E[use]))
        newV = np.where(active, np.minimum(V, cand), V)
        U = newV < V
        V = newV
        out.append((V.copy(), int(active.sum()), int(np.diff(R.astype(np.int64))[active].sum())))
    return out


def check(R, C, E, V0, source):
    a = plain_loop(R, C, E, V0, source, fused=False)
    b = plain_loop(R, C, E, V0, source, fused=True)
    assert len(a) == len(b) and len(a) > 1
    for (va, aa, ea), (vb, ab, eb) in zip(a, b):
        np.testing.assert_array_equal(va, vb)
        assert (aa, ea) == (ab, eb)
    return a[-1][0]


def test_fused_step_matches_plain_cfg1(cfg1_edges):
    s, d, w = cfg1_edges
    hg = O.build_host_graph(s, d, w, init="source", source=0, inf=O.INF32)
    final = check(hg.R, hg.C, hg.E, hg.V, 0)
    want, _ = O.jacobi_fixed_point(hg.R, hg.C, hg.E, hg.V, op=O.OP_SSSP_SAT)
    np.testing.assert_array_equal(final.astype(np.uint32), want)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_fused_step_matches_plain_random(seed):
    rng = np.random.default_rng(seed)
    n, m = 300, 2400
    s = rng.integers(0, n, m).astype(np.uint32)
    d = rng.integers(0, n, m).astype(np.uint32)
    w = rng.integers(1, 50, m).astype(np.uint32)
    keep = s != d
    hg = O.build_host_graph(s[keep], d[keep], w[keep], init="source", source=int(s[0]),
                            inf=O.INF32)
    check(hg.R, hg.C, hg.E, hg.V, int(s[0]))
