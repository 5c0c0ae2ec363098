"""CPU restatement of the FP32 preconditioner's levels (csrc/mg27.cu and the
level-0 transfers) for the GPU tests: FP64 scipy.sparse on dense (z, y, x)
arrays of side n.

  A0       the reference's operator: diagonal D = (deg + pw*screen) (n-1)^2,
           couplings -(n-1)^2 to in-grid face neighbours
  s        prolongation weights: 1 on nodes of the coarse grid (all coordinates
           even), else clip((sum_{j != i} -a_ij) / a_ii, 0, 1)
  P_s      diag(s) P, P trilinear
  A_c      P_s^T A P_s / 8  (27-point)
  restrict R r = P^T (s r) / 8
  relax    red-black ordered sweep, same-colour couplings from the previous iterate
  cycle    V(pre, post) on level 0, coarse_sweeps each way below, 3^3 solved exactly
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def forward_offsets():
    return [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
            if dz > 0 or (dz == 0 and (dy > 0 or (dy == 0 and dx > 0)))]


def fwd_index(dx, dy, dz):
    if dz == 1:
        return 1 + (dy + 1) * 3 + (dx + 1)
    return 10 + (dx + 1) if dy == 1 else 13


def coords(n):
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    return z.ravel(), y.ravel(), x.ravel()


def degree(n):
    z, y, x = coords(n)
    return ((x > 0).astype(int) + (x < n - 1) + (y > 0) + (y < n - 1) + (z > 0) + (z < n - 1)).reshape(n, n, n)


def level0_diagonal(screen, pw):
    n = screen.shape[0]
    h2 = float(n - 1) ** 2
    return (degree(n) + pw * screen) * h2


def operator7(D):
    n = D.shape[0]
    h2 = float(n - 1) ** 2
    one = sp.diags([np.ones(n - 1), np.ones(n - 1)], [-1, 1])
    I = sp.identity(n)
    adj = sp.kron(sp.kron(one, I), I) + sp.kron(sp.kron(I, one), I) + sp.kron(sp.kron(I, I), one)
    return (sp.diags(D.ravel()) - h2 * adj).tocsr()


def weights(A, n):
    d = A.diagonal()
    off = -(np.asarray(A.sum(axis=1)).ravel() - d)
    z, y, x = coords(n)
    on_coarse = ((x | y | z) & 1) == 0
    return np.where(on_coarse, 1.0, np.clip(off / d, 0.0, 1.0))


def trilinear(n):
    cn = (n + 1) // 2
    p = sp.lil_matrix((n, cn))
    for i in range(n):
        if i % 2 == 0:
            p[i, i // 2] = 1.0
        else:
            p[i, i // 2] = 0.5
            p[i, i // 2 + 1] = 0.5
    p = p.tocsr()
    return sp.kron(sp.kron(p, p), p).tocsr()


def galerkin(A, s, n):
    Ps = (sp.diags(s) @ trilinear(n)).tocsr()
    return ((Ps.T @ A @ Ps) / 8.0).tocsr()


def _wt1(d):
    return 1.0 if d == 0 else (0.5 if abs(d) == 1 else 0.0)


def galerkin_separable(A, s, n):
    """P^T (S A S) P / 8 for a 27-point A contracted one axis at a time (x, then
    y, then z), as csrc/mg27.cu's galerkin_x/y/z kernels do: each stage maps
    fine positions 2M + a and offsets d to coarse offsets m with weights
    P(a) P(a + d - 2m), keeping the other two axes' offsets.  Returns the
    coarse operator's 14 planes (plane 0 the diagonal)."""
    cn = (n + 1) // 2
    st = np.zeros((n, n, n, 3, 3, 3))  # st[z, y, x, dz+1, dy+1, dx+1] = s_i a_ij s_j
    coo = A.tocoo()
    z, y, x = coords(n)
    for i, j, a in zip(coo.row, coo.col, coo.data):
        d = (z[j] - z[i], y[j] - y[i], x[j] - x[i])
        if max(abs(v) for v in d) <= 1:
            st[z[i], y[i], x[i], d[0] + 1, d[1] + 1, d[2] + 1] = s[i] * a * s[j]
    b1 = np.zeros((n, n, cn, 3, 3, 3))  # [z, y, I, dz, dy, m]
    for a in (-1, 0, 1):
        xi = 2 * np.arange(cn) + a
        ok = (xi >= 0) & (xi < n)
        for dx in (-1, 0, 1):
            for m in (-1, 0, 1):
                w = _wt1(a) * _wt1(a + dx - 2 * m)
                if w:
                    b1[:, :, ok, :, :, m + 1] += w * st[:, :, xi[ok], :, :, dx + 1]
    b2 = np.zeros((n, cn, cn, 3, 3, 3))  # [z, J, I, dz, my, m]
    for b in (-1, 0, 1):
        yj = 2 * np.arange(cn) + b
        ok = (yj >= 0) & (yj < n)
        for dy in (-1, 0, 1):
            for my in (-1, 0, 1):
                w = _wt1(b) * _wt1(b + dy - 2 * my)
                if w:
                    b2[:, ok, :, :, my + 1, :] += w * b1[:, yj[ok], :, :, dy + 1, :]
    c = np.zeros((cn, cn, cn, 3, 3, 3))  # [K, J, I, mz, my, m]
    for cc in (-1, 0, 1):
        zf = 2 * np.arange(cn) + cc
        ok = (zf >= 0) & (zf < n)
        for dz in (-1, 0, 1):
            for mz in (-1, 0, 1):
                w = _wt1(cc) * _wt1(cc + dz - 2 * mz)
                if w:
                    c[ok, :, :, mz + 1, :, :] += w * b2[zf[ok], :, :, dz + 1, :, :]
    c /= 8.0
    out = np.zeros((14, cn, cn, cn))
    out[0] = c[..., 1, 1, 1]
    for (kx, ky, kz) in forward_offsets():
        out[fwd_index(kx, ky, kz)] = c[..., kz + 1, ky + 1, kx + 1]
    return out


def planes(A, n):
    """14 dense (n, n, n) planes: the diagonal, then a(J, J+K) for forward K."""
    out = np.zeros((14, n, n, n))
    coo = A.tocoo()
    z, y, x = coords(n)
    dz, dy, dx = z[coo.col] - z[coo.row], y[coo.col] - y[coo.row], x[coo.col] - x[coo.row]
    flat = out.reshape(14, -1)
    for k, (ox, oy, oz) in [(0, (0, 0, 0))] + [(fwd_index(*K), K) for K in forward_offsets()]:
        sel = (dx == ox) & (dy == oy) & (dz == oz)
        flat[k, coo.row[sel]] = coo.data[sel]
    return out


def from_planes(pl, n):
    """Symmetric sparse operator from 14 dense planes (inverse of `planes`)."""
    z, y, x = coords(n)
    idx = np.arange(n ** 3)
    rows, cols, vals = [idx], [idx], [pl[0].ravel()]
    for K in forward_offsets():
        dx, dy, dz = K
        ok = (x + dx >= 0) & (x + dx < n) & (y + dy >= 0) & (y + dy < n) & (z + dz >= 0) & (z + dz < n)
        j = idx + dx + dy * n + dz * n * n
        v = pl[fwd_index(*K)].ravel()
        rows += [idx[ok], j[ok]]
        cols += [j[ok], idx[ok]]
        vals += [v[ok], v[ok]]
    return sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n ** 3, n ** 3)).tocsr()


def hierarchy(screen, pw):
    """Operators and weights of every level, finest first (side down to 3)."""
    n = screen.shape[0]
    A = operator7(level0_diagonal(screen, pw))
    ops, ws, sizes = [A], [weights(A, n)], [n]
    while n > 3:
        A = galerkin(A, ws[-1], n)
        n = (n + 1) // 2
        ops.append(A)
        ws.append(weights(A, n))
        sizes.append(n)
    return ops, ws, sizes


def relax(A, e_prev, rhs, n, zero=False):
    d = A.diagonal()
    z, y, x = coords(n)
    colour = (x + y + z) & 1
    prev = np.zeros(n ** 3) if zero else e_prev.ravel().copy()
    nxt = prev.copy()
    b = rhs.ravel()
    for c in (0, 1):
        src = prev if c == 0 else nxt
        new = (b - (A @ src - d * src)) / d
        nxt = np.where(colour == c, new, nxt)
    return nxt.reshape(n, n, n)


def residual_restrict(A, s, e, rhs, n):
    res = s * (rhs.ravel() - A @ e.ravel())
    cn = (n + 1) // 2
    return (trilinear(n).T @ res / 8.0).reshape(cn, cn, cn), res.reshape(n, n, n)


def prolong(fine, coarse, s, n):
    return fine + (s * (trilinear(n) @ coarse.ravel())).reshape(n, n, n)


def v_cycle(ops, ws, sizes, level, rhs, pre=3, post=3, coarse_sweeps=2):
    """The cycle below `level` from a zero start, as the GPU runs it."""
    A, n = ops[level], sizes[level]
    if level > 0:
        pre = post = coarse_sweeps
    if level == len(ops) - 1:
        return np.linalg.solve(A.toarray(), rhs.ravel()).reshape(n, n, n)
    e = relax(A, None, rhs, n, zero=True)
    for _ in range(pre - 1):
        e = relax(A, e, rhs, n)
    coarse_rhs, _ = residual_restrict(A, ws[level], e, rhs, n)
    c = v_cycle(ops, ws, sizes, level + 1, coarse_rhs, pre, post, coarse_sweeps)
    e = prolong(e, c, ws[level], n)
    for _ in range(post):
        e = relax(A, e, rhs, n)
    return e


def packed_offsets():
    """The 26 coupling offsets (dx, dy, dz) of a packed level, plane order."""
    return [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if dx or dy or dz]


def pack(A, n):
    """Per-colour packed couplings (FP16, 26 x n x n x Pc) and 1/diagonal (FP32,
    n x n x Pc) of a 27-point level, as pb_pack27_f32 computes them from FP32
    coefficients: inv = 1/d and c_K = (-a_JK) * inv in FP32, rounded to FP16."""
    pc = (n + 1) // 2
    A = A.tocsr()
    d = A.diagonal().astype(np.float32)
    inv = (np.float32(1.0) / d).astype(np.float32)
    z, y, x = coords(n)
    h = [np.zeros((26, n, n, pc), np.float16) for _ in range(2)]
    iv = [np.zeros((n, n, pc), np.float32) for _ in range(2)]
    dense = {}
    coo = A.tocoo()
    for r, c, v in zip(coo.row, coo.col, coo.data):
        dense[(r, c)] = v
    for j in range(n ** 3):
        col = (x[j] + y[j] + z[j]) & 1
        iv[col][z[j], y[j], x[j] >> 1] = inv[j]
        for k, (dx, dy, dz) in enumerate(packed_offsets()):
            xx, yy, zz = x[j] + dx, y[j] + dy, z[j] + dz
            a = 0.0
            if 0 <= xx < n and 0 <= yy < n and 0 <= zz < n:
                a = dense.get((j, (zz * n + yy) * n + xx), 0.0)
            h[col][k, z[j], y[j], x[j] >> 1] = np.float16(np.float32(-np.float32(a)) * inv[j])
    return h[0], h[1], iv[0], iv[1]


def packed_operator(h0, h1, inv0, inv1, n):
    """The row operator a packed level applies: a_JJ = 1/inv_J, a_JK = -c_K / inv_J."""
    z, y, x = coords(n)
    colour = (x + y + z) & 1
    i = x >> 1
    inv = np.where(colour == 0, inv0[z, y, i], inv1[z, y, i]).astype(np.float64)
    idx = np.arange(n ** 3)
    rows, cols, vals = [idx], [idx], [1.0 / inv]
    for k, (dx, dy, dz) in enumerate(packed_offsets()):
        c = np.where(colour == 0, h0[k, z, y, i], h1[k, z, y, i]).astype(np.float64)
        ok = (x + dx >= 0) & (x + dx < n) & (y + dy >= 0) & (y + dy < n) & (z + dz >= 0) & (z + dz < n) & (c != 0)
        rows.append(idx[ok])
        cols.append(idx[ok] + dx + dy * n + dz * n * n)
        vals.append(-c[ok] / inv[ok])
    return sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n ** 3, n ** 3)).tocsr()
