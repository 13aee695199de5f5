"""wc_eigen against the reference's known answers (spectral/lanczos/tests.rs)
and against dense eigendecompositions (numpy.linalg.eigh) of the same
operator: eigenvalues within 1e-10, residuals ‖Mx − λx‖ ≤ 1e-8."""

import numpy as np
import pytest

import oracle as O
import pg_warren_b200 as W

pytestmark = pytest.mark.gpu


def undirected(n, pairs, weights=None):
    edges = []
    for q, (a, b) in enumerate(pairs):
        w = 1.0 if weights is None else weights[q]
        edges += [(0, a, b, w), (0, b, a, w)]
    og = O.Graph.from_edges(n, edges, weighted=weights is not None)
    off, tgt, w, _, _, _ = og.csr()
    return W.GraphVersion(off, tgt, w), off, tgt, w


def dense_operator(n, off, tgt, w, op):
    a = np.zeros((n, n))
    for i in range(n):
        for e in range(off[i], off[i + 1]):
            a[i, tgt[e]] += 1.0 if w is None else w[e]
    a = (a + a.T) / 2
    d = a.sum(axis=1)
    active = (np.abs(a) > 0).sum(axis=1) > 0
    idx = np.where(active)[0]
    s = a[np.ix_(idx, idx)]
    dd = d[idx]
    if op == "adjacency":
        return s, idx
    if op == "laplacian":
        return np.diag(dd) - s, idx
    inv = 1.0 / np.sqrt(dd)
    if op == "normalized_laplacian":
        return np.eye(len(idx)) - inv[:, None] * s * inv[None, :], idx
    return inv[:, None] * s * inv[None, :], idx


def test_the_smallest_laplacian_eigenpairs_of_a_path():
    # spectral/lanczos/tests.rs:75-98
    n = 60
    gv, *_ = undirected(n, [(i, i + 1) for i in range(n - 1)])
    e = W.eigen(gv, W.EigenOptions(4, which="smallest", operator="laplacian", tol=1e-8))
    assert e.converged and len(e.values) == 4
    for j in range(4):
        exp = 2.0 - 2.0 * np.cos(np.pi * j / n)
        assert abs(e.values[j] - exp) < 1e-9
        assert e.residuals[j] < 1e-7
        exact = np.cos(np.pi * j * (np.arange(n) + 0.5) / n)
        exact /= np.linalg.norm(exact)
        assert abs(abs(np.dot(e.vectors[j], exact)) - 1.0) < 1e-8


def test_inactive_nodes_contribute_nothing():
    # spectral/lanczos/tests.rs:114-129
    gv, *_ = undirected(7, [(i, i + 1) for i in range(4)])
    e = W.eigen(gv, W.EigenOptions(5, which="smallest", operator="laplacian"))
    assert abs(e.values[0]) < 1e-6 and e.values[1] > 0.3
    assert np.all(e.vectors[:, 5:] == 0.0)
    with pytest.raises(W.api.EigenpairCount):
        W.eigen(gv, W.EigenOptions(6, operator="laplacian"))


def test_every_copy_of_a_component_eigenvalue_is_found_exactly():
    # spectral/lanczos/tests.rs:543-566: 30 disjoint 40-cycles.
    pairs = []
    for c in range(30):
        pairs += [(40 * c + i, 40 * c + (i + 1) % 40) for i in range(40)]
    gv, *_ = undirected(1201, pairs)
    for op, which, value in [("laplacian", "smallest", 0.0),
                             ("normalized_laplacian", "smallest", 0.0),
                             ("random_walk", "largest", 1.0)]:
        e = W.eigen(gv, W.EigenOptions(20, which=which, operator=op))
        assert e.converged and e.iterations == 0 and e.components == 30
        for c in range(20):
            assert e.values[c] == value
            assert e.residuals[c] < 1e-6
            exact = np.zeros(1201)
            exact[40 * c: 40 * (c + 1)] = 1.0 / np.sqrt(40)
            assert np.abs(e.vectors[c] - exact).max() < 1e-7


def test_normalised_laplacian_zero_vectors_weigh_by_root_degree():
    # spectral/lanczos/tests.rs:568-595: two stars.
    pairs = [(0, l) for l in (1, 2, 3)] + [(4, 4 + l) for l in range(1, 6)]
    gv, *_ = undirected(10, pairs)
    e = W.eigen(gv, W.EigenOptions(2, which="smallest", operator="normalized_laplacian"))
    for c, (centre, leaves, rows) in enumerate([(0, 3, range(0, 4)), (4, 5, range(4, 10))]):
        exact = np.zeros(10)
        for i in rows:
            exact[i] = np.sqrt(leaves) if i == centre else 1.0
        exact /= np.linalg.norm(exact)
        assert e.values[c] == 0.0
        assert np.abs(e.vectors[c] - exact).max() < 1e-15


@pytest.mark.parametrize("op,which", [("adjacency", "largest"), ("laplacian", "smallest"),
                                      ("laplacian", "largest"),
                                      ("normalized_laplacian", "smallest"),
                                      ("normalized_laplacian", "largest"),
                                      ("random_walk", "largest")])
def test_eigenvalues_match_a_dense_decomposition(op, which):
    rng = np.random.default_rng(17)
    n = 300
    pairs = {(int(a), int(b)) for a, b in rng.integers(0, n, (900, 2)) if a != b}
    pairs = sorted(pairs)
    weights = list(rng.uniform(0.5, 2.0, len(pairs)))
    gv, off, tgt, w = undirected(n, pairs, weights)
    k = 6
    e = W.eigen(gv, W.EigenOptions(k, which=which, operator=op, tol=1e-13, max_iter=20000))
    m, idx = dense_operator(n, off, tgt, w, op)
    lam = np.linalg.eigvalsh(m)
    if which == "smallest":
        exp = np.sort(lam)[:k]
    else:
        order = sorted(range(len(lam)), key=lambda i: (-abs(lam[i]), -lam[i]))
        exp = lam[order[:k]]
    assert np.abs(np.sort(e.values) - np.sort(exp)).max() < 1e-10 * max(1.0, np.abs(lam).max())
    assert e.residuals.max() <= 1e-8


def test_rmat_largest_component_normalised_laplacian_smallest():
    # The C4 workload's shape at a size a dense solve can check: the
    # symmetrised R-MAT's largest component, 16 smallest eigenpairs.
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components
    g = W.rmat(11, undirected=True)
    n = g.id_space
    rows = np.repeat(np.arange(n), np.diff(g.offsets).astype(np.int64))
    a = csr_matrix((np.ones(g.edges), (rows, g.targets)), shape=(n, n))
    _, labels = connected_components(a, directed=False)
    big = np.bincount(labels).argmax()
    keep = np.where(labels == big)[0]
    sub = a[keep][:, keep].tocsr()
    sub.sort_indices()
    gv = W.GraphVersion(sub.indptr.astype(np.uint64), sub.indices.astype(np.uint32))
    e = W.eigen(gv, W.EigenOptions(16, which="smallest", operator="normalized_laplacian",
                                   tol=1e-13, max_iter=100000, seed=3))
    d = np.asarray(sub.sum(axis=1)).ravel()
    inv = 1.0 / np.sqrt(d)
    m = np.eye(len(keep)) - inv[:, None] * sub.toarray() * inv[None, :]
    lam = np.sort(np.linalg.eigvalsh(m))[:16]
    assert e.components == 1 and e.exact == 1
    assert np.abs(e.values - lam).max() < 1e-10
    assert e.residuals.max() <= 1e-8


def _largest_component(scale):
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components
    g = W.rmat(scale, undirected=True)
    n = g.id_space
    rows = np.repeat(np.arange(n), np.diff(g.offsets).astype(np.int64))
    a = csr_matrix((np.ones(g.edges), (rows, g.targets)), shape=(n, n))
    _, labels = connected_components(a, directed=False)
    keep = np.where(labels == np.bincount(labels).argmax())[0]
    sub = a[keep][:, keep].tocsr()
    sub.sort_indices()
    return sub


def test_rmat16_largest_component_matches_an_independent_solver():
    # The C4 variant's shape at R-MAT 16 (46,777 nodes): the 16 smallest
    # eigenvalues of the normalised Laplacian against ARPACK (scipy's
    # eigsh) on 2I - L, whose largest eigenvalues are 2 minus those.
    from scipy.sparse import diags, identity
    from scipy.sparse.linalg import eigsh
    sub = _largest_component(16)
    gv = W.GraphVersion(sub.indptr.astype(np.uint64), sub.indices.astype(np.uint32))
    e = W.eigen(gv, W.EigenOptions(16, which="smallest", operator="normalized_laplacian",
                                   tol=1e-13, max_iter=100000, seed=3))
    inv = diags(1.0 / np.sqrt(np.asarray(sub.sum(axis=1)).ravel()))
    m = identity(sub.shape[0]) + inv @ sub @ inv
    lam = np.sort(2.0 - eigsh(m, k=16, which="LA", ncv=96, tol=1e-14, maxiter=100000,
                              return_eigenvectors=False))
    assert e.components == 1 and e.exact == 1
    assert np.abs(np.sort(e.values) - lam).max() < 1e-10
    assert e.residuals.max() <= 1e-8
