"""The device colouring's argument, checked on the CPU.

ufc_pattern_build colours the elements by sweeping the map
colour[e] = mex{colour[f] : f < e shares a node with e} over all elements in
parallel, in place, from colour 0, until a sweep changes nothing.  The
sequential greedy colouring of RT_AsmColor_Build (the oracle's
orc_color_elements) is that map's only fixed point, so any order of updates
that settles reaches it.  Here the sweeps are restated in numpy with two
extreme update orders -- all elements at once from the previous sweep's
colours (Jacobi), and in-place in a random order per sweep (the GPU's blocks
run in no fixed order) -- and both must end on the oracle's colouring; the
sweep counts show the nx + ny + nz growth on lexicographically numbered
boxes that the device's sweep limit is sized for."""
import numpy as np
import pytest


def _lower_lists(conn, n_nodes):
    E = conn.shape[0]
    by_node = [[] for _ in range(n_nodes)]
    for e in range(E):
        for nd in conn[e]:
            by_node[nd].append(e)
    lower = []
    for e in range(E):
        s = set()
        for nd in conn[e]:
            s.update(f for f in by_node[nd] if f < e)
        lower.append(np.array(sorted(s), dtype=np.int64))
    return lower


def _mex(colours):
    used = set(colours.tolist())
    c = 0
    while c in used:
        c += 1
    return c


def _sweeps(lower, order_rng=None, max_sweeps=10000):
    E = len(lower)
    col = np.zeros(E, dtype=np.int64)
    for s in range(1, max_sweeps + 1):
        if order_rng is None:  # Jacobi: every element reads the previous sweep
            new = np.array([_mex(col[lower[e]]) for e in range(E)])
            changed = not np.array_equal(new, col)
            col = new
        else:  # in place, random order
            changed = False
            for e in order_rng.permutation(E):
                c = _mex(col[lower[e]])
                if c != col[e]:
                    col[e] = c
                    changed = True
        if not changed:
            return col, s
    raise AssertionError("sweeps did not settle")


def _shuffle(conn, seed):
    return np.ascontiguousarray(conn[np.random.default_rng(seed).permutation(conn.shape[0])])


@pytest.mark.parametrize("dims,shuffle", [((6, 3, 3), None), ((10, 4, 3), None), ((6, 3, 3), 5), ((30, 1, 1), None)])
def test_sweeps_reach_the_sequential_greedy_colouring(pkg, orc, dims, shuffle):
    p = pkg.mesh.cantilever(*dims, float(dims[0]), float(dims[1]), float(dims[2]))
    conn = p.conn if shuffle is None else _shuffle(p.conn, shuffle)
    ref, ncol = orc.color_elements(p.n_nodes, conn)
    lower = _lower_lists(np.asarray(conn), p.n_nodes)
    col_j, sweeps_j = _sweeps(lower)
    col_r, _ = _sweeps(lower, np.random.default_rng(1))
    assert np.array_equal(col_j, ref) and np.array_equal(col_r, ref)
    assert col_j.max() + 1 == ncol
    if shuffle is None:
        # lexicographic boxes: about nx + ny + nz sweeps (the last one changes nothing)
        assert sweeps_j <= sum(dims) + 3, sweeps_j
