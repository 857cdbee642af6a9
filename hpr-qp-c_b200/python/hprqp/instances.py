"""Seeded synthetic QP instances for tests and benchmarks.

The reference measures on a private MPS corpus that is not available, so these
generators stand in for it.  Each recipe follows the five workload
descriptions of this project (plain n=1000 QP, large power-law QP,
factor-structured portfolio, 4096-instance batch, 256-instance
differentiation batch).  Every instance is built from
``numpy.random.default_rng(0x48505251 + 1000 * config + instance)`` so a
(config, instance) pair always produces the same arrays on any machine.

All matrices are returned as ``QPInstance`` with 0-based CSR arrays
(``indptr`` int64, ``indices`` int64, ``data`` float64), Q given as a full
symmetric matrix (the builder symmetrises it again, which leaves it
unchanged).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

SEED_BASE = 0x48505251


@dataclass
class CSR:
    nrow: int
    ncol: int
    indptr: np.ndarray
    indices: np.ndarray
    data: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.data, self.indices, self.indptr), shape=(self.nrow, self.ncol))

    def dense(self) -> np.ndarray:
        out = np.zeros((self.nrow, self.ncol))
        for r in range(self.nrow):
            s, e = self.indptr[r], self.indptr[r + 1]
            np.add.at(out[r], self.indices[s:e], self.data[s:e])
        return out


@dataclass
class QPInstance:
    Q: CSR
    A: CSR
    c: np.ndarray
    AL: np.ndarray
    AU: np.ndarray
    l: np.ndarray
    u: np.ndarray
    obj_constant: float = 0.0
    name: str = ""

    @property
    def n(self) -> int:
        return self.Q.ncol

    @property
    def m(self) -> int:
        return self.A.nrow


def _csr_from_coo(nrow: int, ncol: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray) -> CSR:
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    indptr = np.zeros(nrow + 1, dtype=np.int64)
    np.add.at(indptr, rows + 1, 1)
    np.cumsum(indptr, out=indptr)
    return CSR(nrow, ncol, indptr, cols.astype(np.int64), vals.astype(np.float64))


def _csr_from_scipy(mat) -> CSR:
    mat = mat.tocsr()
    mat.sum_duplicates()
    mat.sort_indices()
    return CSR(mat.shape[0], mat.shape[1], mat.indptr.astype(np.int64), mat.indices.astype(np.int64),
               mat.data.astype(np.float64))


def _uniform_pattern(rng: np.random.Generator, nrow: int, ncol: int, nnz: int):
    """nnz distinct positions drawn uniformly without replacement."""
    total = nrow * ncol
    nnz = min(nnz, total)
    flat = rng.choice(total, size=nnz, replace=False)
    flat.sort()
    return (flat // ncol).astype(np.int64), (flat % ncol).astype(np.int64)


def _gram_plus_ridge(rng: np.random.Generator, n: int, k: int, density: float, ridge: float) -> CSR:
    """Q = M'M + ridge*I with M k x n, the given density, N(0,1) values."""
    import scipy.sparse as sp

    nnz_m = max(1, int(round(density * k * n)))
    r, c = _uniform_pattern(rng, k, n, nnz_m)
    M = sp.csr_matrix((rng.standard_normal(len(r)), (r, c)), shape=(k, n))
    Q = (M.T @ M).tocsr() + ridge * sp.identity(n, format="csr")
    return _csr_from_scipy(Q)


def _feasible_rows(rng: np.random.Generator, A: CSR, n: int, n_eq: int):
    x0 = rng.uniform(-1.0, 1.0, n)
    r = A.to_scipy() @ x0
    AL = r.copy()
    AU = r.copy()
    rest = A.nrow - n_eq
    if rest > 0:
        AL[n_eq:] = r[n_eq:] - rng.uniform(0.0, 1.0, rest)
        AU[n_eq:] = r[n_eq:] + rng.uniform(0.0, 1.0, rest)
    return AL, AU


def plain_qp(seed: int, n: int = 1000, m: int = 500, a_density: float = 0.01,
             m_rows: int = 200, m_density: float = 0.005, n_eq: int = 300,
             bound: float = 10.0, name: str = "") -> QPInstance:
    """The plain single-QP recipe (n=1000, m=500 at the defaults)."""
    rng = np.random.default_rng(seed)
    r, c = _uniform_pattern(rng, m, n, int(round(a_density * m * n)))
    A = _csr_from_coo(m, n, r, c, rng.standard_normal(len(r)))
    Q = _gram_plus_ridge(rng, n, m_rows, m_density, 0.01)
    cvec = rng.standard_normal(n)
    AL, AU = _feasible_rows(rng, A, n, n_eq)
    l = np.full(n, -bound)
    u = np.full(n, bound)
    return QPInstance(Q, A, cvec, AL, AU, l, u, 0.0, name or f"plain_n{n}_m{m}")


def config0(instance: int = 0) -> QPInstance:
    return plain_qp(SEED_BASE + instance, name="config0")


def config1(instance: int = 0, scale: float = 1.0) -> QPInstance:
    """Large power-law QP: n=1e6, m=5e5, nnz(A)~1e7 Zipf(1.5) rows clipped to
    [1,5000]; Q = diag U(0.1,10) + B'B with B 2e5 x 1e6 and 2.5e6 nnz.
    ``scale`` shrinks every dimension (for tests)."""
    import scipy.sparse as sp

    rng = np.random.default_rng(SEED_BASE + 1000 + instance)
    n = int(round(1_000_000 * scale))
    m = int(round(500_000 * scale))
    target = 10_000_000 * scale
    raw = rng.zipf(1.5, m).astype(np.float64)
    raw = np.minimum(raw, 5000.0)
    lens = np.clip(np.rint(raw * (target / raw.sum())), 1, min(5000, n)).astype(np.int64)
    total = int(lens.sum())
    rows = np.repeat(np.arange(m, dtype=np.int64), lens)
    cols = rng.integers(0, n, total, dtype=np.int64)
    key = np.unique(rows * n + cols)  # drop the rare duplicate column within a row
    rows, cols = key // n, key % n
    A = _csr_from_coo(m, n, rows, cols, rng.standard_normal(len(rows)))
    kb = int(round(200_000 * scale))
    nnz_b = int(round(2_500_000 * scale))
    br = rng.integers(0, kb, nnz_b, dtype=np.int64)
    bc = rng.integers(0, n, nnz_b, dtype=np.int64)
    B = sp.csr_matrix((rng.standard_normal(nnz_b), (br, bc)), shape=(kb, n))
    Q = (B.T @ B).tocsr() + sp.diags(rng.uniform(0.1, 10.0, n), format="csr")
    Qc = _csr_from_scipy(Q)
    cvec = rng.standard_normal(n)
    AL, AU = _feasible_rows(rng, A, n, int(0.4 * m))
    return QPInstance(Qc, A, cvec, AL, AU, np.full(n, -10.0), np.full(n, 10.0), 0.0, "config1")


def config1_sized_plain(instance: int = 0, scale: float = 1.0) -> QPInstance:
    """The plain recipe (uniform A pattern, Q = M'M + 0.01 I, x in [-10, 10],
    40% equality rows) at the large QP's sizes: n=1e6, m=5e5, nnz(A)=1e7,
    M 2e5 x 1e6 with 2.5e6 nnz (nnz(Q) ~ 3.2e7).  Used for the single large
    backward, whose forward solve must reach its tolerance.  Positions are
    drawn with replacement and duplicates dropped (a few per million)."""
    import scipy.sparse as sp

    rng = np.random.default_rng(SEED_BASE + 5000 + instance)
    n = int(round(1_000_000 * scale))
    m = int(round(500_000 * scale))
    nnz_a = int(round(10_000_000 * scale))
    key = np.unique(rng.integers(0, m, nnz_a, dtype=np.int64) * n + rng.integers(0, n, nnz_a, dtype=np.int64))
    A = _csr_from_coo(m, n, key // n, key % n, rng.standard_normal(len(key)))
    kb = int(round(200_000 * scale))
    nnz_b = int(round(2_500_000 * scale))
    bkey = np.unique(rng.integers(0, kb, nnz_b, dtype=np.int64) * n + rng.integers(0, n, nnz_b, dtype=np.int64))
    M = sp.csr_matrix((rng.standard_normal(len(bkey)), (bkey // n, bkey % n)), shape=(kb, n))
    Q = _csr_from_scipy((M.T @ M).tocsr() + 0.01 * sp.identity(n, format="csr"))
    cvec = rng.standard_normal(n)
    AL, AU = _feasible_rows(rng, A, n, int(0.4 * m))
    return QPInstance(Q, A, cvec, AL, AU, np.full(n, -10.0), np.full(n, 10.0), 0.0, "config1_sized_plain")


def config2(instance: int = 0, n_assets: int = 200_000, k: int = 200, sectors: int = 500) -> QPInstance:
    """Factor-structured portfolio QP with variables (x, f), f = F'x."""
    rng = np.random.default_rng(SEED_BASE + 2000 + instance)
    n = n_assets + k
    D = rng.uniform(0.01, 0.1, n_assets)
    qd = np.concatenate([2.0 * D, np.full(k, 2.0)])
    Q = CSR(n, n, np.arange(n + 1, dtype=np.int64), np.arange(n, dtype=np.int64), qd)
    F = rng.normal(0.0, 0.1, (n_assets, k))
    sector_of = rng.integers(0, sectors, n_assets)
    m = k + 1 + sectors
    # factor rows: F[:,j]' x - f_j = 0
    fr_ptr = np.arange(k + 1, dtype=np.int64) * (n_assets + 1)
    fr_idx = np.empty(k * (n_assets + 1), dtype=np.int64)
    fr_val = np.empty(k * (n_assets + 1))
    for j in range(k):
        s = j * (n_assets + 1)
        fr_idx[s:s + n_assets] = np.arange(n_assets)
        fr_val[s:s + n_assets] = F[:, j]
        fr_idx[s + n_assets] = n_assets + j
        fr_val[s + n_assets] = -1.0
    # stable sort keeps asset indices increasing inside each sector row
    order = np.argsort(sector_of, kind="stable")
    counts = np.bincount(sector_of, minlength=sectors)
    indptr = np.concatenate([fr_ptr, [fr_ptr[-1] + n_assets],
                             fr_ptr[-1] + n_assets + np.cumsum(counts)]).astype(np.int64)
    indices = np.concatenate([fr_idx, np.arange(n_assets), order.astype(np.int64)])
    data = np.concatenate([fr_val, np.ones(n_assets), np.ones(n_assets)])
    A = CSR(m, n, indptr, indices, data)
    AL = np.concatenate([np.zeros(k), [1.0], np.full(sectors, -0.05)])
    AU = np.concatenate([np.zeros(k), [1.0], np.full(sectors, 0.05)])
    cvec = np.concatenate([rng.normal(0.0005, 0.01, n_assets), np.zeros(k)])
    l = np.concatenate([np.zeros(n_assets), np.full(k, -np.inf)])
    u = np.concatenate([np.full(n_assets, 0.01), np.full(k, np.inf)])
    return QPInstance(Q, A, cvec, AL, AU, l, u, 0.0, "config2")


def config3_instance(instance: int) -> QPInstance:
    """One member of the 4096-instance batch: n~U{50..2000}, m~U{ceil(n/4)..n},
    A density U(0.5%,5%), Q = M'M + 0.01 I with M n/5 x n sized so that
    nnz(Q) ~ dQ n^2, dQ ~ U(0.1%, 2%); 60% equality rows."""
    rng = np.random.default_rng(SEED_BASE + 3000 + instance)
    n = int(rng.integers(50, 2001))
    m = int(rng.integers(-(-n // 4), n + 1))
    dA = rng.uniform(0.005, 0.05)
    dQ = rng.uniform(0.001, 0.02)
    k = max(1, n // 5)
    m_density = min(1.0, float(np.sqrt(5.0 * dQ / n)))
    sub_seed = int(rng.integers(0, 2**62))
    return plain_qp(sub_seed, n=n, m=m, a_density=dA, m_rows=k, m_density=m_density,
                    n_eq=int(0.6 * m), name=f"config3_{instance}")


def config3(count: int = 4096, start: int = 0) -> List[QPInstance]:
    return [config3_instance(start + i) for i in range(count)]


def config4_instance(instance: int) -> QPInstance:
    return plain_qp(SEED_BASE + 4000 + instance, n=500, m=300, n_eq=150, name=f"config4_{instance}")


def config4(count: int = 256, start: int = 0) -> List[QPInstance]:
    return [config4_instance(start + i) for i in range(count)]


def adjoint_case(instance: int, n: int = 60, m: int = 30) -> QPInstance:
    """Small QP with bounds tight enough that a share of variables and rows
    end at a bound (for differentiation tests): box [-0.5, 0.5] on most
    variables, a few free variables, equality, ranged and one-sided rows."""
    rng = np.random.default_rng(SEED_BASE + 5000 + instance)
    r, c = _uniform_pattern(rng, m, n, int(0.15 * m * n))
    A = _csr_from_coo(m, n, r, c, rng.standard_normal(len(r)))
    Q = _gram_plus_ridge(rng, n, n // 2, 0.1, 0.1)
    x0 = rng.uniform(-0.3, 0.3, n)
    ax = A.to_scipy() @ x0
    n_eq = m // 4
    AL = ax - rng.uniform(0.0, 0.5, m)
    AU = ax + rng.uniform(0.0, 0.5, m)
    AL[:n_eq] = AU[:n_eq] = ax[:n_eq]
    one_sided = rng.random(m) < 0.25
    one_sided[:n_eq] = False
    AU[one_sided] = np.inf
    l = np.full(n, -0.5)
    u = np.full(n, 0.5)
    free = rng.random(n) < 0.1
    l[free], u[free] = -np.inf, np.inf
    cvec = 3.0 * rng.standard_normal(n)
    return QPInstance(Q, A, cvec, AL, AU, l, u, 0.0, f"adjoint_{instance}")


@dataclass
class SOCInstance:
    """A QP with second-order cones: the QPInstance data plus cone offsets
    (variables [var_offsets[0], n), rows [row_offsets[0], m)) and rhs."""
    qp: QPInstance
    var_offsets: Optional[np.ndarray]
    row_offsets: Optional[np.ndarray]
    rhs: Optional[np.ndarray]


def soc_case(instance: int, n_lin: int = 20, cone: int = 6, m_lin: int = 6, row_cone: int = 4) -> SOCInstance:
    """min 1/2 x'Dx + c'x + t  s.t.  (t, v) in K (a variable cone), v = Bx - d,
    random ranged rows on x, |Cx - e| <= rho (a row cone: A_K x - rhs in K),
    x in [-1, 1]; D diagonal U(0.5, 2)."""
    rng = np.random.default_rng(SEED_BASE + 6000 + instance)
    k = max(cone - 1, 0)
    n = n_lin + cone
    x0 = rng.uniform(-0.5, 0.5, n_lin)
    B = rng.standard_normal((k, n_lin)) * (rng.random((k, n_lin)) < 0.5)
    d = rng.standard_normal(k)
    G = rng.standard_normal((m_lin, n_lin)) * (rng.random((m_lin, n_lin)) < 0.4)
    rc = max(row_cone - 1, 0)
    C = rng.standard_normal((rc, n_lin)) * (rng.random((rc, n_lin)) < 0.5)
    e = rng.standard_normal(rc)
    rho = float(np.linalg.norm(C @ x0 - e)) + 0.5
    rows, AL, AU, rhs = [], [], [], []
    for j in range(k):  # v_j - (B x)_j = -d_j
        r = np.zeros(n)
        r[:n_lin] = -B[j]
        r[n_lin + 1 + j] = 1.0
        rows.append(r)
        AL.append(-d[j])
        AU.append(-d[j])
        rhs.append(0.0)
    gx = G @ x0
    for j in range(m_lin):
        r = np.zeros(n)
        r[:n_lin] = G[j]
        rows.append(r)
        AL.append(gx[j] - rng.uniform(0.1, 1.0))
        AU.append(gx[j] + rng.uniform(0.1, 1.0))
        rhs.append(0.0)
    m_lin_total = len(rows)
    if row_cone:
        rows.append(np.zeros(n))  # cone head: 0 - (-rho) = rho
        rhs.append(-rho)
        for j in range(rc):
            r = np.zeros(n)
            r[:n_lin] = C[j]
            rows.append(r)
            rhs.append(e[j])
        AL += [-np.inf] * row_cone
        AU += [np.inf] * row_cone
    Adense = np.array(rows)
    rr, cc = np.nonzero(Adense)
    A = _csr_from_coo(Adense.shape[0], n, rr.astype(np.int64), cc.astype(np.int64), Adense[rr, cc])
    qd = np.concatenate([rng.uniform(0.5, 2.0, n_lin), np.zeros(cone)])
    nzq = np.nonzero(qd)[0]
    Q = _csr_from_coo(n, n, nzq.astype(np.int64), nzq.astype(np.int64), qd[nzq])
    cvec = np.concatenate([rng.standard_normal(n_lin), [1.0] if cone else [], np.zeros(k)])
    l = np.concatenate([np.full(n_lin, -1.0), np.full(cone, -np.inf)])
    u = np.concatenate([np.full(n_lin, 1.0), np.full(cone, np.inf)])
    qp = QPInstance(Q, A, cvec, np.array(AL), np.array(AU), l, u, 0.0, f"soc_{instance}")
    return SOCInstance(qp, np.array([n_lin, n], np.int64) if cone else None,
                       np.array([m_lin_total, m_lin_total + row_cone], np.int64) if row_cone else None,
                       np.array(rhs) if row_cone else None)


def tiny_cases() -> List[QPInstance]:
    """Hand-written models mirroring the reference's test fixtures
    (tests/test_support.c:79-268 of the reference project): dense-list form
    converted to CSR."""
    inf = np.inf

    def dense(Qd, Ad, c, AL, AU, l, u, name):
        Qd = np.asarray(Qd, dtype=float)
        n = Qd.shape[0]
        Ad = np.asarray(Ad, dtype=float).reshape(-1, n)

        def to_csr(M):
            rows, cols = np.nonzero(M)
            return _csr_from_coo(M.shape[0], M.shape[1], rows.astype(np.int64), cols.astype(np.int64), M[rows, cols])

        return QPInstance(to_csr(Qd), to_csr(Ad), np.asarray(c, float), np.asarray(AL, float),
                          np.asarray(AU, float), np.asarray(l, float), np.asarray(u, float), 0.0, name)

    return [
        dense([[2, 0], [0, 4]], [[1, 1]], [2, 1], [2], [2], [0, 0], [10, 10], "standard"),
        dense([[2, 0], [0, 4]], [[1, 1]], [2, 1], [2], [2], [-inf, -inf], [inf, inf], "standard_noC"),
        dense([[4, 0], [0, 9]], [[16, 25]], [2, 4], [2], [6], [0, -1], [10, 3], "scale"),
        dense([[2, 0], [0, 4]], [[1, 2]], [1, -1], [0], [100], [0, 0], [10, 10], "residuals"),
        dense([[2, 1], [1, 2]], [[1, 2]], [0, 0], [-1], [1], [-10, -10], [10, 10], "dense_q"),
        dense([[2, 0.5], [0.5, 3]], [[1, -1]], [1, -0.5], [0], [1.5], [-10, -10], [10, 10], "control_nondiag"),
        dense([[2, 0], [0, 3]], np.zeros((0, 2)), [1, -0.5], [], [], [-inf, -inf], [inf, inf], "empty_a"),
        dense([[3, 0], [0, 5]], [[1, 1], [1, -1], [2, 0.5]], [1.5, -0.5], [1, -0.5, 0.25], [1, -0.5, 0.25],
              [0, -1], [2, 3], "tall_diag"),
        dense([[1]], np.zeros((0, 1)), [0], [], [], [-1], [1], "dispatch_1d"),
        dense([[2]], [[3]], [0], [-1], [1], [-10], [10], "gpu_spmv_1d"),
        dense([[2, 0.5], [0.5, 3]], [[1, -2]], [0.5, -0.25], [-0.5], [0.75], [-1, -1], [1, 1], "iteration_standard"),
        dense([[0]], np.zeros((0, 1)), [0], [], [], [-1], [1], "zero_1d"),
    ]
