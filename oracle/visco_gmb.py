"""CPU restatement of the reference's generalized-Maxwell-body fit of visco-elastic media, in the
reference's own arithmetic (float storage, the terms its pow() calls promote in double).

TEST INFRASTRUCTURE: only tests/ use it, as the checker of cgfd_visco_gmb (which solves the same
least-squares problem in FP64); it is never part of the product path. Parity: pinned by
tests/test_gpu_visco.py, which checks the product's fit against the reference's own
md_vis_GMB_cal_Y built unmodified (oracle/_ref/ref_harness).

Follows md_t.cu:657-781 (md_vis_GMB_cal_Y), md_t.cu:783-850 (md_visco_LS: the normal equations
(G^T G)^-1 G^T d with d = Q^-1 in every row) and md_t.cu:852-914 (md_visco_LS_mat_inv: Gauss-Jordan
elimination, a row swap only on a zero pivot). PI is constants.h's 3.1415926535898.
"""
import numpy as np

PI = 3.1415926535898
f32 = np.float32


def _mat_inv(a):
    """md_visco_LS_mat_inv on an n x n float matrix: returns the inverse (float)."""
    n = a.shape[0]
    m = a.astype(f32).copy()
    inv = np.eye(n, dtype=f32)
    for k in range(n):
        if m[k, k] == 0:
            j = next((jj for jj in range(k + 1, n) if m[jj, k] != 0), n)
            if j == n:
                raise ValueError("matrix is not invertible")
            m[[k, j]] = m[[j, k]]
            inv[[k, j]] = inv[[j, k]]
        t = m[k, k]
        m[k] = m[k] / t
        inv[k] = inv[k] / t
        for i in range(n):
            if i == k:
                continue
            t = m[i, k]
            m[i] = m[i] - m[k] * t
            inv[i] = inv[i] - inv[k] * t
    return inv


def _ls(g, d):
    """md_visco_LS: Y = (G^T G)^-1 G^T (d, ..., d), accumulated in float."""
    gt = g.T.astype(f32)
    mul = np.zeros((g.shape[1], g.shape[1]), f32)
    for i in range(g.shape[1]):
        for j in range(g.shape[1]):
            acc = f32(0)
            for k in range(g.shape[0]):
                acc = f32(acc + gt[i, k] * g[k, j])
            mul[i, j] = acc
    inv = _mat_inv(mul)
    m2 = np.zeros_like(gt)
    for i in range(gt.shape[0]):
        for j in range(gt.shape[1]):
            acc = f32(0)
            for k in range(gt.shape[0]):
                acc = f32(acc + inv[i, k] * gt[k, j])
            m2[i, j] = acc
    out = np.zeros(gt.shape[0], f32)
    for i in range(gt.shape[0]):
        acc = f32(0)
        for j in range(gt.shape[1]):
            acc = f32(acc + m2[i, j] * f32(d))
        out[i] = acc
    return out


def gmb_fit(visco, lam, mu, qp, qs):
    """md_vis_GMB_cal_Y over arrays of points. Returns (lam_u, mu_u, Ylam [nmax, n], Ymu [nmax, n],
    wl [nmax]) as float32."""
    nm = int(visco["nmaxwell"])
    kmax = 2 * nm - 1
    wr = f32(2 * PI * f32(visco["fr"]))
    wmin = f32(2 * PI * f32(visco["fmin"]))
    wmax = f32(2 * PI * f32(visco["fmax"]))
    wratio = f32(wmax / wmin)
    wk = np.array([f32(wmin * (float(wratio) ** (k / f32(kmax - 1)))) if kmax > 1 else wmin for k in range(kmax)], f32)
    wl = wk[0::2][:nm].astype(f32)
    lam, mu, qp, qs = (np.ravel(np.asarray(a, f32)) for a in (lam, mu, qp, qs))
    n = lam.size
    lu, mu_u = np.zeros(n, f32), np.zeros(n, f32)
    yl, ym = np.zeros((nm, n), f32), np.zeros((nm, n), f32)
    cache = {}

    def fit(q):
        q1 = f32(1.0 / round(float(q)))
        if float(q1) not in cache:
            g = np.array([[f32((float(wl[j] * wk[m]) + float(wl[j]) ** 2 * float(q1)) /
                               (float(wl[j]) ** 2 + float(wk[m]) ** 2)) for j in range(nm)] for m in range(kmax)], f32)
            y = _ls(g, q1)
            t = f32(0)
            for j in range(nm):
                t = f32(t + y[j] / (1 + (float(wr) / float(wl[j])) ** 2))
            th1 = f32(1 - t)
            t = f32(0)
            for j in range(nm):
                t = f32(t + y[j] * wr / wl[j] / (1 + (float(wr) / float(wl[j])) ** 2))
            th2 = t
            r = f32(np.sqrt(float(th1) ** 2 + float(th2) ** 2))
            cache[float(q1)] = (y, th1, r)
        return cache[float(q1)]

    for t in range(n):
        yp, th1p, rp = fit(qp[t])
        ys, th1s, rs = fit(qs[t])
        kappa = f32((lam[t] + 2 * mu[t]) * (rp + th1p) / (2 * float(rp) ** 2))
        m_u = f32(mu[t] * (rs + th1s) / (2 * float(rs) ** 2))
        mu_u[t] = m_u
        lu[t] = f32(kappa - 2 * m_u)
        for j in range(nm):
            yl[j, t] = f32((1 + 2 * m_u / lu[t]) * yp[j] - 2 * m_u / lu[t] * ys[j])
            ym[j, t] = ys[j]
    return lu, mu_u, yl, ym, wl
