"""Seeded synthetic SDP instances in HDSDP's user-data layout.

An SDP block is handed to ``HUserDataSetConeData`` as a CSC matrix with
``n(n+1)/2`` rows and ``m+1`` columns (interface/def_hdsdp_user_data.h:11-21):
column 0 holds the objective C, column i the constraint matrix A_i, and the
row index of the lower-triangle entry (i, j), i >= j, is
``PACK_IDX(n, i, j) = (2n - j - 1) j / 2 + i`` (interface/hdsdp_utils.h:49).
An off-diagonal packed entry stands for the symmetric pair (i, j) and (j, i).

The problem solved is ``min <C, X>  s.t.  <A_i, X> = b_i,  X psd``.

Each generator follows one workload of the benchmark suite; they are seeded
stand-ins for public instances (no benchmark data is shipped).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def pack_idx(n: int, i, j):
    """Packed lower-triangle row index of entry (i, j) with i >= j."""
    i = np.asarray(i, dtype=np.int64)
    j = np.asarray(j, dtype=np.int64)
    return ((2 * n - j - 1) * j) // 2 + i


@dataclass
class SDPInstance:
    """One dense SDP block plus the right-hand side, in the reference layout."""

    name: str
    n: int
    m: int
    Ap: np.ndarray  # int32, m + 2
    Ai: np.ndarray  # int32, nnz
    Ax: np.ndarray  # float64, nnz
    b: np.ndarray   # float64, m
    meta: dict = field(default_factory=dict)

    def column(self, k: int):
        """(packed row indices, values) of column k (0 = C, k = A_k)."""
        s, e = int(self.Ap[k]), int(self.Ap[k + 1])
        return self.Ai[s:e], self.Ax[s:e]

    def dense(self, k: int) -> np.ndarray:
        """Column k expanded to a full symmetric n x n matrix (small n only)."""
        n = self.n
        rows, vals = self.column(k)
        # invert PACK_IDX column by column
        M = np.zeros((n, n))
        starts = pack_idx(n, np.arange(n), np.arange(n))
        j = np.searchsorted(starts, rows, side="right") - 1
        i = rows - starts[j] + j
        M[i, j] = vals
        M[j, i] = vals
        return M


def _assemble(name, n, cols, b, meta=None) -> SDPInstance:
    """cols: list of (packed_idx, values) for C, A_1..A_m."""
    m = len(cols) - 1
    Ap = np.zeros(m + 2, dtype=np.int64)
    idx_parts, val_parts = [], []
    for k, (idx, val) in enumerate(cols):
        idx = np.asarray(idx, dtype=np.int64)
        val = np.asarray(val, dtype=np.float64)
        order = np.argsort(idx, kind="stable")
        idx, val = idx[order], val[order]
        if idx.size > 1 and np.any(np.diff(idx) == 0):
            raise ValueError("duplicate packed entries in column %d" % k)
        idx_parts.append(idx)
        val_parts.append(val)
        Ap[k + 1] = Ap[k] + idx.size
    Ai = np.concatenate(idx_parts) if idx_parts else np.zeros(0, np.int64)
    Ax = np.concatenate(val_parts) if val_parts else np.zeros(0)
    if Ai.size and Ai.max() >= n * (n + 1) // 2:
        raise ValueError("packed index out of range")
    return SDPInstance(name, n, m, Ap.astype(np.int32), Ai.astype(np.int32),
                       Ax.astype(np.float64), np.asarray(b, dtype=np.float64), meta or {})


def _laplacian_objective(n, ei, ej, w):
    """C = -L/4 for the weighted graph (ei > ej), packed lower triangle."""
    deg = np.zeros(n)
    np.add.at(deg, ei, w)
    np.add.at(deg, ej, w)
    diag_idx = pack_idx(n, np.arange(n), np.arange(n))
    keep = deg != 0
    idx = np.concatenate([diag_idx[keep], pack_idx(n, ei, ej)])
    val = np.concatenate([-deg[keep] / 4.0, w / 4.0])
    return idx, val


def _erdos_renyi_edges(n, p, rng):
    iu = np.tril_indices(n, -1)
    mask = rng.random(iu[0].size) < p
    return iu[0][mask].astype(np.int64), iu[1][mask].astype(np.int64)


def maxcut(n: int = 200, p: float = 0.05, seed: int = 1, n_edges: int | None = None,
           weights: tuple | None = None) -> SDPInstance:
    """MaxCut SDP relaxation: min <-L/4, X> s.t. diag(X) = 1.

    With ``n_edges`` set, that many distinct edges are drawn uniformly (the
    large sparse case); otherwise G(n, p). Weights are 1, or U(lo, hi).
    """
    rng = np.random.default_rng(seed)
    if n_edges is None:
        ei, ej = _erdos_renyi_edges(n, p, rng)
    else:
        picks = set()
        while len(picks) < n_edges:
            u = rng.integers(0, n, size=2 * (n_edges - len(picks)) + 16)
            v = rng.integers(0, n, size=u.size)
            for a, c in zip(u.tolist(), v.tolist()):
                if a == c:
                    continue
                picks.add((max(a, c), min(a, c)))
                if len(picks) == n_edges:
                    break
        pairs = np.array(sorted(picks), dtype=np.int64)
        ei, ej = pairs[:, 0], pairs[:, 1]
    if weights is None:
        w = np.ones(ei.size)
    else:
        w = rng.uniform(weights[0], weights[1], size=ei.size)
    cols = [_laplacian_objective(n, ei, ej, w)]
    for i in range(n):
        cols.append(([pack_idx(n, i, i)], [1.0]))
    b = np.ones(n)
    return _assemble("maxcut", n, cols, b, {"edges": int(ei.size), "seed": seed})


def lovasz_theta(n: int = 300, p: float = 0.1, seed: int = 2) -> SDPInstance:
    """Lovasz theta SDP: min <-J, X> s.t. tr(X) = 1, X_ij = 0 for edges ij."""
    rng = np.random.default_rng(seed)
    ei, ej = _erdos_renyi_edges(n, p, rng)
    inst = lovasz_theta_graph(n, list(zip(ei.tolist(), ej.tolist())))
    inst.meta["seed"] = seed
    return inst


def lovasz_theta_graph(n: int, edges) -> SDPInstance:
    """Lovasz theta SDP of a given graph; ``edges`` lists pairs (a, c) with a > c.

    Known answers: theta(C_5) = sqrt(5), theta(K_n) = 1, theta(empty graph on n) = n.
    """
    ei = np.array([e[0] for e in edges], dtype=np.int64)
    ej = np.array([e[1] for e in edges], dtype=np.int64)
    npack = n * (n + 1) // 2
    cols = [(np.arange(npack), -np.ones(npack))]
    cols.append((pack_idx(n, np.arange(n), np.arange(n)), np.ones(n)))
    for a, c in zip(ei.tolist(), ej.tolist()):
        cols.append(([pack_idx(n, a, c)], [1.0]))
    b = np.zeros(1 + ei.size)
    b[0] = 1.0
    return _assemble("theta", n, cols, b, {"edges": int(ei.size)})


def rank_one(n: int = 1000, m: int = 2000, density: float = 0.1, seed: int = 3) -> SDPInstance:
    """Random rank-one SDP: A_i = a_i a_i^T with a fixed support size.

    X0 = I + G G^T / n (G is n x 20) is primal feasible, b_i = a_i^T X0 a_i,
    and C = I + R with R symmetric, 1% of off-diagonal pairs U(-0.1, 0.1),
    so the dual is strictly feasible.
    """
    rng = np.random.default_rng(seed)
    k = max(1, int(round(density * n)))
    G = rng.standard_normal((n, 20))
    cols = []
    # objective
    iu = np.tril_indices(n, -1)
    mask = rng.random(iu[0].size) < 0.01
    ri, rj = iu[0][mask], iu[1][mask]
    rv = rng.uniform(-0.1, 0.1, size=ri.size)
    cidx = np.concatenate([pack_idx(n, np.arange(n), np.arange(n)), pack_idx(n, ri, rj)])
    cval = np.concatenate([np.ones(n), rv])
    cols.append((cidx, cval))
    b = np.zeros(m)
    for t in range(m):
        supp = np.sort(rng.choice(n, size=k, replace=False))
        a = rng.standard_normal(k)
        # lower triangle of a a^T on the support
        I, J = np.tril_indices(k)
        cols.append((pack_idx(n, supp[I], supp[J]), a[I] * a[J]))
        Ga = G[supp].T @ a
        b[t] = a @ a + Ga @ Ga / n
    return _assemble("rank_one", n, cols, b, {"support": k, "seed": seed})


def theta_adjoint(n: int = 200, p: float = 0.1, zero_frac: float = 0.2, seed: int = 5) -> SDPInstance:
    """Theta-style SDP for the differentiable layer.

    min <-W, X> s.t. tr(X) = 1 and X_ij = 0 on a seeded ``zero_frac`` subset of
    the non-edges; W symmetric on the edge support with U(0, 1) entries.
    """
    rng = np.random.default_rng(seed)
    ei, ej = _erdos_renyi_edges(n, p, rng)
    w = rng.uniform(0.0, 1.0, size=ei.size)
    edge = np.zeros((n, n), dtype=bool)
    edge[ei, ej] = True
    iu = np.tril_indices(n, -1)
    non = ~edge[iu]
    ni, nj = iu[0][non], iu[1][non]
    pick = rng.random(ni.size) < zero_frac
    zi, zj = ni[pick], nj[pick]
    cols = [(pack_idx(n, ei, ej), -w)]
    cols.append((pack_idx(n, np.arange(n), np.arange(n)), np.ones(n)))
    for a, c in zip(zi.tolist(), zj.tolist()):
        cols.append(([pack_idx(n, a, c)], [1.0]))
    b = np.zeros(1 + zi.size)
    b[0] = 1.0
    return _assemble("theta_adjoint", n, cols, b,
                     {"edges": int(ei.size), "zeros": int(zi.size), "seed": seed})


def _dense_columns(n, mats):
    """(packed index, value) columns of full symmetric matrices (their nonzero lower entries)."""
    ii, jj = np.tril_indices(n)
    idx = pack_idx(n, ii, jj)
    cols = []
    for M in mats:
        v = M[ii, jj]
        keep = v != 0
        cols.append((idx[keep], v[keep]))
    return cols


def dense_coeff(n: int = 80, m: int = 40, seed: int = 21) -> SDPInstance:
    """SDP whose constraint matrices are general dense symmetric matrices (full rank).

    A_i = (R_i + R_i^T) / 2 with R_i Gaussian, so the presolve keeps them dense
    (interface/hdsdp_sdpdata.c:2273) and the Schur rows take the dense-coefficient
    path. X0 = I + G G^T / n (G n x 5) is primal feasible with b_i = <A_i, X0>,
    and C = I + 0.1 (Q + Q^T) / (2 sqrt(n)) is positive definite, so y = 0 is a
    strictly feasible dual point.
    """
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, 5))
    X0 = np.eye(n) + G @ G.T / n
    Q = rng.standard_normal((n, n))
    C = np.eye(n) + 0.1 * (Q + Q.T) / (2.0 * np.sqrt(n))
    mats, b = [C], np.zeros(m)
    for t in range(m):
        R = rng.standard_normal((n, n))
        A = (R + R.T) / 2.0
        mats.append(A)
        b[t] = float(np.sum(A * X0))
    return _assemble("dense_coeff", n, _dense_columns(n, mats), b, {"seed": seed})


def dual_infeasible(n: int = 8, seed: int = 1) -> SDPInstance:
    """An SDP with no dual feasible point, which sends the infeasible-start method into
    the homogeneous self-dual embedding (interface/hdsdp_algo.c:1866-1870).

    C = -I + 0.05 (G + G^T) with G Gaussian is negative definite, and only the first
    n/2 diagonal entries are constrained (X_ii = 1), so C - sum_i y_i e_i e_i^T is
    never positive semidefinite and the primal  min <C, X>  is unbounded.
    """
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n)) * 0.05
    mats = [-np.eye(n) + G + G.T]
    for i in range(n // 2):
        E = np.zeros((n, n))
        E[i, i] = 1.0
        mats.append(E)
    return _assemble("dual_infeasible", n, _dense_columns(n, mats), np.ones(n // 2), {"seed": seed})


def lp_block(m: int, n_lp: int, per_col: int = 2, seed: int = 7):
    """An LP cone for an instance with m constraints, in the user CSC layout the LP cone
    takes (interface/hdsdp_conic_lp.c:99-158): column 0 the costs c (U(0.5, 1.5)),
    column i the coefficients of constraint i on the LP columns. Each LP column k gets
    `per_col` constraints with U(0.2, 1) coefficients, so s = c - A^T y > 0 for every
    y <= 0; returns (n_lp, Ap, Ai, Ax)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.5, 1.5, size=n_lp)
    cols = [[] for _ in range(m)]
    for k in range(n_lp):
        for i in rng.choice(m, size=min(per_col, m), replace=False):
            cols[int(i)].append((k, float(rng.uniform(0.2, 1.0))))
    Ap, Ai, Ax = [0], [], []
    for k in range(n_lp):
        Ai.append(k)
        Ax.append(float(c[k]))
    Ap.append(len(Ai))
    for i in range(m):
        for k, v in sorted(cols[i]):
            Ai.append(k)
            Ax.append(v)
        Ap.append(len(Ai))
    return n_lp, np.asarray(Ap, np.int32), np.asarray(Ai, np.int32), np.asarray(Ax, np.float64)


@dataclass
class ConicProblem:
    """Several cones sharing one set of m constraints, in the user layout: ``cones`` lists
    (kind, dim, Ap, Ai, Ax) with kind "sdp" (a block of order dim, packed lower-triangle
    rows) or "lp" (dim columns), each a CSC matrix with m + 1 columns, column 0 the cone's
    objective. The problem is  min sum_k <C_k, X_k>  s.t.  sum_k <A_ik, X_k> = b_i."""

    name: str
    m: int
    b: np.ndarray
    cones: list
    meta: dict = field(default_factory=dict)

    def sdp_block(self, k: int) -> SDPInstance:
        """Cone k (an SDP block) as an SDPInstance with this problem's right-hand side."""
        kind, n, Ap, Ai, Ax = self.cones[k]
        assert kind == "sdp"
        return SDPInstance("%s[%d]" % (self.name, k), n, self.m, Ap, Ai, Ax, self.b)


def _csc_columns(m, cols):
    """CSC arrays from per-column (rows, values) lists (None = empty column), rows sorted."""
    Ap, Ai, Ax = [0], [], []
    for c in cols:
        if c is not None:
            idx = np.asarray(c[0], dtype=np.int64)
            val = np.asarray(c[1], dtype=np.float64)
            o = np.argsort(idx, kind="stable")
            Ai.extend(idx[o].tolist())
            Ax.extend(val[o].tolist())
        Ap.append(len(Ai))
    return np.asarray(Ap, np.int32), np.asarray(Ai, np.int32), np.asarray(Ax, np.float64)


def multiblock(dims, m_local, m_couple: int, n_lp: int = 0, seed: int = 11, name: str = "multiblock") -> ConicProblem:
    """SDP blocks of orders ``dims`` (an optional LP cone of ``n_lp`` columns last) with
    ``m_local[k]`` constraints on block k alone and ``m_couple`` constraints on every block.

    Coefficients are unit diagonals e_i e_i^T, edges E_ac + E_ca, sparse rank-one a a^T
    (support 3) and sparse symmetric matrices, distinct within a block. C_k = I + R_k with a
    few off-diagonal entries of size <= 0.1, and the LP costs are U(0.5, 1.5), so y = 0 is
    strictly dual feasible; b = A(X0) at X0_k = I + G_k G_k^T / n_k (G_k n_k x 3) and the LP
    point x0 = 1, so the primal is strictly feasible too.
    """
    rng = np.random.default_rng(seed)
    K = len(dims)
    m = int(sum(m_local)) + int(m_couple)
    cols = [[None] * (m + 1) for _ in range(K)]
    X0 = []
    for k, n in enumerate(dims):
        idx = [int(pack_idx(n, i, i)) for i in range(n)]
        val = [1.0] * n
        for _ in range(n // 2):
            if n < 2:
                break
            a, c = sorted(rng.choice(n, size=2, replace=False).tolist(), reverse=True)
            p = int(pack_idx(n, a, c))
            if p not in idx:
                idx.append(p)
                val.append(float(rng.uniform(-0.1, 0.1)))
        cols[k][0] = (idx, val)
        G = rng.standard_normal((n, 3))
        X0.append(np.eye(n) + G @ G.T / n)

    def coeff(n, seen):
        for _ in range(100):
            t = 0 if n == 1 else int(rng.integers(0, 4))
            if t == 0:
                i = int(rng.integers(0, n))
                ent = {(i, i): 1.0}
            elif t == 1:
                a, c = sorted(rng.choice(n, size=2, replace=False).tolist(), reverse=True)
                ent = {(a, c): 1.0}
            elif t == 2:
                sup = np.sort(rng.choice(n, size=min(3, n), replace=False))
                av = rng.standard_normal(sup.size)
                ent = {}
                for p in range(sup.size):
                    for q in range(p + 1):
                        ent[(int(sup[p]), int(sup[q]))] = float(av[p] * av[q])
            else:
                i = int(rng.integers(0, n))
                ent = {(i, i): float(rng.uniform(0.5, 2.0))}
                for _ in range(2):
                    a, c = sorted(rng.choice(n, size=2, replace=False).tolist(), reverse=True)
                    ent[(a, c)] = float(rng.uniform(-1.0, 1.0))
            key = tuple(sorted((k2, round(v, 12)) for k2, v in ent.items()))
            if key not in seen:
                seen.add(key)
                return ent
        raise ValueError("block of order %d cannot hold that many distinct constraints" % n)

    def add(k, row, ent):
        n = dims[k]
        idx = [int(pack_idx(n, a, c)) for (a, c) in ent]
        val = list(ent.values())
        cols[k][row + 1] = (idx, val)
        return sum((v if a == c else 2.0 * v) * X0[k][a, c] for (a, c), v in ent.items())

    b = np.zeros(m)
    row = 0
    for k, n in enumerate(dims):
        seen = set()
        for _ in range(m_local[k]):
            b[row] = add(k, row, coeff(n, seen))
            row += 1
    for _ in range(m_couple):
        for k, n in enumerate(dims):
            b[row] += add(k, row, coeff(n, set()))
        row += 1
    cones = []
    for k, n in enumerate(dims):
        Ap, Ai, Ax = _csc_columns(m, cols[k])
        cones.append(("sdp", int(n), Ap, Ai, Ax))
    if n_lp > 0:
        c = rng.uniform(0.5, 1.5, size=n_lp)
        lcols = [None] * (m + 1)
        lcols[0] = (list(range(n_lp)), c.tolist())
        per = [dict() for _ in range(m)]
        for q in range(n_lp):
            for i in rng.choice(m, size=min(2, m), replace=False):
                v = float(rng.uniform(-1.0, 1.0))
                per[int(i)][q] = v
                b[int(i)] += v  # x0 = 1
        for i in range(m):
            if per[i]:
                lcols[i + 1] = (list(per[i].keys()), list(per[i].values()))
        Ap, Ai, Ax = _csc_columns(m, lcols)
        cones.append(("lp", int(n_lp), Ap, Ai, Ax))
    return ConicProblem(name, m, b, cones, {"dims": list(map(int, dims)), "m_local": list(map(int, m_local)),
                                            "m_couple": int(m_couple), "n_lp": int(n_lp), "seed": seed})


# Multi-cone parity cases: all dense cones; dense and sparse cones with a 1 x 1 block; two
# dense cones and an LP cone; a larger mixed case.
MULTIBLOCK_CASES = {
    "mb3": dict(dims=[20, 15, 10], m_local=[25, 20, 15], m_couple=6, seed=11),
    "mb5_sparse": dict(dims=[12, 10, 8, 6, 1], m_local=[10, 8, 6, 4, 1], m_couple=3, seed=12),
    "mb2_lp": dict(dims=[30, 25], m_local=[30, 30], m_couple=5, n_lp=12, seed=13),
    "mb4_n500": dict(dims=[200, 150, 100, 50], m_local=[300, 200, 150, 100], m_couple=50, seed=14),
    # six sparse cones (each holds at most 26 % of the rows) and no dense or LP cone: the
    # reference takes its sparse Schur complement here (interface/hdsdp_schur.c:181-254)
    "mb6_sparse": dict(dims=[30, 25, 20, 20, 15, 10], m_local=[40, 35, 30, 30, 25, 20], m_couple=8, seed=15),
    # 40 sparse cones of order 60 with 120 constraints each and 40 shared ones (m = 4,840):
    # the Schur complement is a block arrow with 40 blocks of 120 rows and 40 coupling rows
    "mb40_arrow": dict(dims=[60] * 40, m_local=[120] * 40, m_couple=40, seed=16),
}


# Multi-block problems too large for the compiled reference (its sparse KKT goes through a
# dense stand-in here) and for a dense Schur matrix on one GPU: 250 sparse cones of order 90
# with 450 constraints each and 100 shared ones, m = 112,600, whose dense M and factor would
# take 203 GB. The block arrow holds 250 blocks of 450 rows and 100 coupling rows.
LARGE_ARROW_CASES = {
    "mb250_m112k": dict(dims=[90] * 250, m_local=[450] * 250, m_couple=100, seed=17),
    # the same family at 60 cones (m = 27,100), small enough for a dense M as well
    "mb60_m27k": dict(dims=[90] * 60, m_local=[450] * 60, m_couple=100, seed=18),
}


def multiblock_case(name: str) -> ConicProblem:
    spec = MULTIBLOCK_CASES.get(name) or LARGE_ARROW_CASES[name]
    return multiblock(name=name, **spec)


WORKLOADS = {
    "maxcut_n200": lambda: maxcut(200, 0.05, seed=1),
    "theta_n300": lambda: lovasz_theta(300, 0.1, seed=2),
    "rank1_n1000_m2000": lambda: rank_one(1000, 2000, 0.1, seed=3),
    "maxcut_n8000": lambda: maxcut(8000, seed=4, n_edges=40000, weights=(0.5, 1.5)),
    "theta_adjoint_n200": lambda: theta_adjoint(200, 0.1, 0.2, seed=5),
    # the n = 2000 layer with 2 % of the non-edges fixed to zero (m about 39,600; the 20 %
    # subset of the full-size layer would need a 1.25 TB dense Schur matrix)
    "theta_adjoint_n2000_r2": lambda: theta_adjoint(2000, 0.01, 0.02, seed=6),
}
