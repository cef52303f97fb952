"""TEST INFRASTRUCTURE -- CPU restatement of the reference hot path (the oracle).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this module, and only as the checker; the product never calls it.

Each function restates one reference routine of f-fathurrahman/ffr-pspw-dft-c in
numpy/scipy FP64, citing the file:line it follows.  Arrays keep the reference's
Fortran (column-major) layouts; complex arrays are complex128.

A *cell* here is a dict with the basis and potential arrays the reference keeps
in its globals (common_pspw.h:43-148) for one k-point (ik=1):

    nr      (NR1, NR2, NR3)
    n123    uint32[NGWX]     1-based linear FFT-grid index (GkVectorsGen.cpp:379)
    xkg     float64[NGWX]    |k+G|^2 in (2pi/ALAT)^2 units
    eigr    complex[NGWX, NAX, NSP]  (Fortran order)
    pkg_a   float64[NLMAX, NGWX, NSP]
    wnl     float64[NSP, NLMAX]
    na      int[NSP]
    lm_end  int[NSP]         L_MAX^2 - 2 L_LOC + 1  (ApplyHam_block.cpp:69)
    tpiba2, alat, omega
"""
from __future__ import annotations

import numpy as np
import scipy.linalg.lapack as lapack

# ---------------------------------------------------------------- FFT

def _grid_view(flat, nr):
    n1, n2, n3 = nr
    return flat.reshape(n3, n2, n1)  # Fortran (i1,i2,i3) == C (i3,i2,i1)


def fft_inverse(flat, nr):
    """fft_fftw3.cpp:13-46, inverse=true: FFTW_BACKWARD (exponent +i), unscaled."""
    g = _grid_view(flat, nr)
    return (np.fft.ifftn(g) * g.size).reshape(-1)


def fft_forward(flat, nr):
    """fft_fftw3.cpp:13-46, inverse=false: FFTW_FORWARD (exponent -i), then 1/N."""
    g = _grid_view(flat, nr)
    return (np.fft.fftn(g) / g.size).reshape(-1)


# ---------------------------------------------------------------- H*psi

def projectors(cell, ngw):
    """The KB projectors beta_p(G) = EIGR(G,a) * PKG_A(lm,G) and weights W_p,
    enumerated species-major, then atom, then lm (ApplyHam_block.cpp:68-117).

    Returns (beta[ngw, nproj] complex, w[nproj])."""
    cols, ws = [], []
    for s in range(len(cell["na"])):
        for a in range(cell["na"][s]):
            for lm in range(cell["lm_end"][s]):
                cols.append(cell["eigr"][:ngw, a, s] * cell["pkg_a"][lm, :ngw, s])
                ws.append(cell["wnl"][s, lm])
    if not cols:
        return np.zeros((ngw, 0), complex), np.zeros(0)
    return np.stack(cols, axis=1), np.asarray(ws, dtype=float)


def apply_ham_block(cell, vin, veff, nstates=None):
    """ApplyHam_block.cpp:5-172.  vin: complex[ngw, nstates] (ld = ngw)."""
    vin = np.asarray(vin, dtype=complex)
    if vin.ndim == 1:
        vin = vin[:, None]
    ngw = vin.shape[0]
    if nstates is None:
        nstates = vin.shape[1]
    nr = cell["nr"]
    nnr = nr[0] * nr[1] * nr[2]
    if veff.size != nnr:
        raise ValueError("nnr != NNR")  # ApplyHam_block.cpp:18-21 aborts
    if np.any(np.asarray(cell["lm_end"]) > 4):
        raise ValueError("lm_end > 4 is not implemented")  # :70-73
    idx = cell["n123"][:ngw].astype(np.int64) - 1
    kin = 0.5 * cell["xkg"][:ngw] * cell["tpiba2"]
    beta, w = projectors(cell, ngw)
    vout = np.empty((ngw, nstates), dtype=complex)
    for ist in range(nstates):
        c = np.zeros(nnr, dtype=complex)
        c[idx] = vin[:, ist]                      # :33-36
        c = fft_inverse(c, nr)                    # :41
        c = veff * c                              # :46-48
        c = fft_forward(c, nr)                    # :53
        vout[:, ist] = kin * vin[:, ist] + c[idx]  # :58-61
    # nonlocal part (:68-165): zdotu with conj(EIGR)*PKG_A, back-projection
    # with EIGR*PKG_A -- i.e. beta * W * beta^H * vin.
    if beta.shape[1]:
        p = w[:, None] * (beta.conj().T @ vin[:, :nstates])
        vout += beta @ p
    return vout


def apply_ham(cell, v, veff):
    """ApplyHam.cpp:5-142 (one vector)."""
    return apply_ham_block(cell, np.asarray(v)[:, None], veff)[:, 0]


# ---------------------------------------------------------------- filter

def chebyfilt(cell, X, degree, lb, ub, veff):
    """chebyfilt.cpp:6-74.  Returns the filtered block (X is not modified)."""
    e = (ub - lb) / 2.0
    c = (ub + lb) / 2.0
    sigma = e / (lb - ub)
    sigma1 = sigma
    X = np.array(X, dtype=complex, copy=True)
    Y = apply_ham_block(cell, X, veff)            # :26
    Y = (Y - c * X) * (sigma1 / e)                # :36-39
    for _ in range(2, degree + 1):                # :41-67
        sigma2 = 1.0 / (2.0 / sigma1 - sigma)
        Y1 = apply_ham_block(cell, Y, veff)
        Y1 = Y1 * (2.0 * sigma2 / e)
        Y1 = Y1 + (-c * 2.0 * sigma2 / e) * Y
        Y1 = Y1 + (-sigma * sigma2) * X
        X = Y
        Y = Y1
        sigma = sigma2
    return Y


def chebyfilt_step_coeffs(degree, lb, ub):
    """The scalar coefficients of chebyfilt.cpp:26-67 per degree step d:
    (a, b, c) with Y_d = a*H*Y_{d-1} + b*Y_{d-1} + c*Y_{d-2}, Y_0 = X."""
    e = (ub - lb) / 2.0
    cc = (ub + lb) / 2.0
    sigma = e / (lb - ub)
    sigma1 = sigma
    out = [(sigma1 / e, -cc * sigma1 / e, 0.0)]
    for _ in range(2, degree + 1):
        sigma2 = 1.0 / (2.0 / sigma1 - sigma)
        out.append((2.0 * sigma2 / e, -cc * 2.0 * sigma2 / e, -sigma * sigma2))
        sigma = sigma2
    return out


# ---------------------------------------------------------------- Lanczos

def lanczos(cell, v0, k, veff):
    """lanczos.cpp:8-101.  Returns (T[k,k] real Fortran-layout matrix, f)."""
    v0 = np.array(v0, dtype=complex, copy=True)
    ngw = v0.size
    T = np.zeros((k, k))
    V = np.zeros((ngw, k), dtype=complex)
    h = np.zeros(k, dtype=complex)
    s = np.zeros(k, dtype=complex)
    v0 = v0 / np.sqrt(np.vdot(v0, v0).real)
    V[:, 0] = v0
    Hv = apply_ham(cell, V[:, 0], veff)
    h[0] = np.vdot(V[:, 0], Hv)
    T[0, 0] = h[0].real
    f = Hv - h[0] * V[:, 0]
    s[0] = np.vdot(V[:, 0], f)
    h[0] = h[0] + s[0]
    f = f - s[0] * V[:, 0]
    for j in range(1, k):
        nf = np.vdot(f, f).real
        T[j, j - 1] = np.sqrt(nf)
        V[:, j] = f * (1.0 / np.sqrt(nf))
        Hv = apply_ham(cell, V[:, j], veff)
        f = Hv.copy()
        for i in range(j + 1):
            h[i] = np.vdot(V[:, i], Hv)
            f = f - h[i] * V[:, i]
        for i in range(j + 1):
            s[i] = np.vdot(V[:, i], f)
        h[: j + 1] += s[: j + 1]
        for i in range(j + 1):
            f = f - s[i] * V[:, i]
        T[: j + 1, j] = h[: j + 1].real
    return T, f


def induced_norm_mat(T):
    """ChebySCFLoop.cpp:7-34: || T * (1/sqrt(N)) 1 ||^2."""
    n = T.shape[0]
    v = T @ np.full(n, 1.0 / np.sqrt(n))
    return float(v @ v)


# ---------------------------------------------------------------- random start

_LCG_TABLES: list[np.ndarray] = []


def _lcg_next(a):
    return ((a * 214013 + 2531011) >> 16) & 32767


def _lcg_tables():
    if not _LCG_TABLES:
        f = _lcg_next(np.arange(32768, dtype=np.int64))
        _LCG_TABLES.append(f)
        for _ in range(40):
            f = f[f]
            _LCG_TABLES.append(f)
    return _LCG_TABLES


def random_col(nelem, seed):
    """util_random_cpu.cpp:5-23: LCG a <- ((a*214013+2531011)>>16)&32767;
    each value is ((a mod 100)+1)/a with the *updated* state a, re then im."""
    L = 2 * nelem
    first = _lcg_next(int(seed))  # the seed itself may exceed the table range
    tabs = _lcg_tables()
    t = np.arange(L, dtype=np.int64)  # state after t+1 steps = F^t(first)
    st = np.full(L, first, dtype=np.int64)
    k = 0
    while (1 << k) <= L:
        m = ((t >> k) & 1).astype(bool)
        st[m] = tabs[k][st[m]]
        k += 1
    with np.errstate(divide="ignore", invalid="ignore"):
        vals = ((st % 100) + 1).astype(float) / st.astype(float)
    return vals[0::2] + 1j * vals[1::2]


# ---------------------------------------------------------------- dense LA

def ortho_qr(X):
    """ortho_qr.cpp:3-34: zgeqrf + zungqr (Householder QR, explicit Q)."""
    X = np.asfortranarray(np.array(X, dtype=complex, copy=True))
    m, n = X.shape
    qr, tau, _, info = lapack.zgeqrf(X, lwork=max(1, n))
    if info != 0:
        raise RuntimeError(f"zgeqrf info={info}")
    q, _, info = lapack.zungqr(qr, tau, lwork=max(1, n))
    if info != 0:
        raise RuntimeError(f"zungqr info={info}")
    return q[:, :n]


def eig_zheevd(A):
    """eig_zheevd.cpp:5-34: zheevd('V','U').  Returns (eigenvalues, vectors)."""
    w, v, info = lapack.zheevd(np.asfortranarray(A), compute_v=1, lower=0)
    if info != 0:
        raise RuntimeError(f"zheevd info={info}")
    return w, v


SMALL_ZHEGV = 12.220446049250313e-16  # eig_zhegv.cpp:7


def eig_zhegv_eval(A, B):
    """eig_zhegv.cpp:86-161 (and eig_zhegv 5-83, which discards eval):
    eigendecompose B, scale its vectors by 1/sqrt(eval) where eval > SMALL
    (others left unscaled), A' = S^H (A S), eig(A'), back-transform.
    Returns (eval of A', evec, number of independent vectors)."""
    w, S = eig_zheevd(B)
    S = S.copy()
    nn = 0
    for i in range(S.shape[1]):
        if w[i] > SMALL_ZHEGV:
            nn += 1
            S[:, i] *= 1.0 / np.sqrt(w[i])
    evec = A @ S
    Ap = S.conj().T @ evec
    lam, U = eig_zheevd(Ap)
    return lam, S @ U, nn


def symmetrize(v, ncol=None):
    """lobpcg_cpu.cpp:15-27 over the leading ncol x ncol block: for i <= j,
    v(i,j) = (v(i,j) + conj(v(j,i)))/2 and v(j,i) = conj(v(i,j)).  Every pair
    is visited once, so the result equals (V + V^H)/2 entry by entry."""
    v = np.array(v, copy=True)
    n = v.shape[1] if ncol is None else ncol
    b = v[:n, :n]
    v[:n, :n] = 0.5 * (b + b.conj().T)
    return v


def gen_prec(xkg, alat, tpiba2, tau):
    """GenPrec.cpp:5-24."""
    xkg = np.asarray(xkg, dtype=float)
    if tau <= 0.0:
        x = xkg * (2.0 * np.pi / alat) ** 2
        y = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x))
        return y / (y + 16.0 * x * x * x * x)
    return tau / (0.5 * (xkg + 1.0) * tpiba2)


# ---------------------------------------------------------------- solvers

def _max_iter(nstates, user_max=None):
    if user_max is not None:
        return user_max
    return max(30, nstates // 2)


def davidson(cell, nbasis, nstates, veff, prec, nempty, max_iter=None):
    """davidson_cpu.cpp:9-266.  Returns (evals, X, res_tol)."""
    X = np.stack([random_col(nbasis, 100 + i) for i in range(nstates)], axis=1)  # :47-51
    X = ortho_qr(X)                                                            # :53
    HX = apply_ham_block(cell, X, veff)                                        # :56
    evals = np.einsum("gi,gi->i", X.conj(), HX).real                           # :59-62
    R = evals[None, :] * X - HX                                                # :65-72
    res_tol = np.sqrt(np.einsum("gi,gi->i", R.conj(), R).real)
    max_dir = _max_iter(nstates, max_iter)
    machine_zero = 2.220446049250313e-16
    TOL = 1.0e-6
    n2 = 2 * nstates
    for istep in range(1, max_dir + 1):
        res_norm = np.where(res_tol > machine_zero, 1.0 / np.where(res_tol > 0, res_tol, 1), 1.0)
        R = R * res_norm[None, :]                                              # :96-98
        R = prec[:nbasis, None] * R                                            # :101-105
        HR = apply_ham_block(cell, R, veff)                                    # :118
        h = np.zeros((n2, n2), dtype=complex)
        if istep == 1:
            h[:nstates, :nstates] = X.conj().T @ HX                            # :123
        else:
            h[:nstates, :nstates] = np.diag(evals)                             # :127-132
        h[:nstates, nstates:] = X.conj().T @ HR                                # :138
        h[nstates:, :nstates] = HR.conj().T @ X                                # :141
        h[nstates:, nstates:] = R.conj().T @ HR                                # :146
        o = np.zeros((n2, n2), dtype=complex)
        o[:nstates, :nstates] = np.eye(nstates)                                # :160-165
        o[:nstates, nstates:] = X.conj().T @ R                                 # :169
        o[nstates:, :nstates] = R.conj().T @ X                                 # :172
        o[nstates:, nstates:] = R.conj().T @ R                                 # :177
        lam, evec, _ = eig_zhegv_eval(h, o)                                    # :181
        evals = lam[:nstates].copy()                                           # :184
        c1 = evec[:nstates, :nstates]
        c2 = evec[nstates:, :nstates]
        X = X @ c1 + R @ c2                                                    # :189-204
        HX = HX @ c1 + HR @ c2                                                 # :196-207
        R = evals[None, :] * X - HX                                            # :210-217
        res_tol = np.sqrt(np.einsum("gi,gi->i", R.conj(), R).real)
        nconv = int(np.sum(res_tol < TOL))
        if nconv >= nstates - nempty:
            break
        if np.mean(res_tol) < TOL / 10.0:
            break
    return evals, X, res_tol


def lobpcg(cell, nbasis, nstates, veff, prec, nempty, max_iter=None):
    """lobpcg_cpu.cpp:31-395.  Returns (lambda, X, resnrm)."""
    TOL = 1.0e-6
    TFUDGE = 1.0e10
    maxiter = _max_iter(nstates, max_iter)
    nb = nstates
    X = np.stack([random_col(nbasis, 100 + i) for i in range(nb)], axis=1)    # :82-86
    X = ortho_qr(X)                                                            # :90
    HX = apply_ham_block(cell, X, veff)                                        # :95
    P = HP = None

    def chol_orth(W, HW):
        C = symmetrize(W.conj().T @ W)
        L = np.linalg.cholesky(C)  # C = L L^H, U = L^H
        Ui = np.linalg.inv(L.conj().T)
        return W @ Ui, HW @ Ui

    it = 1
    while True:
        t1 = X.conj().T @ HX                                                   # :103 / :224
        W = HX - X @ t1                                                        # :107-111
        lam, _ = eig_zheevd(t1)                                                # :113
        resnrm = np.sqrt(np.einsum("gi,gi->i", W.conj(), W).real)
        nconv = int(np.sum(resnrm < TOL))
        rnorm = float(np.mean(resnrm))
        if nconv >= nstates - nempty or rnorm < TOL:
            break
        W = prec[:nbasis, None] * W                                            # :142-146
        HW = apply_ham_block(cell, W, veff)                                    # :149
        W, HW = chol_orth(W, HW)                                               # :153-180
        if it == 1:
            Q = np.concatenate([X, W], axis=1)
            HQ = np.concatenate([HX, HW], axis=1)
        else:
            Q = np.concatenate([X, W, P], axis=1)
            HQ = np.concatenate([HX, HW, HP], axis=1)
        T = symmetrize(Q.conj().T @ HQ)                                        # :183-185
        G = symmetrize(Q.conj().T @ Q)                                         # :189-191
        _, U, _ = eig_zhegv_eval(T, G)                                         # :196
        Un = U[:, :nb]
        Xn = Q @ Un
        HXn = HQ @ Un
        if it == 1:
            P, HP = W.copy(), HW.copy()                                        # :211-213
        else:
            P = W @ Un[nb:2 * nb] + P @ Un[2 * nb:3 * nb]                      # :328-335
            HP = HW @ Un[nb:2 * nb] + HP @ Un[2 * nb:3 * nb]                  # :338-345
            P, HP = chol_orth(P, HP)                                           # :348-370
        X, HX = Xn, HXn
        it += 1
        if it > maxiter:
            # the loop (:218) runs iter=2..maxiter and leaves after the
            # rotation of the last iteration without a new check
            break
    return lam, X, resnrm


# ---------------------------------------------------------------- density

def eval_rho_psi(cell, eigvec_flat, ld, ngw, nx, focc, wkpt, omega, ngwx):
    """EvalRhoPsi.cpp:83-157.  eigvec_flat is the caller's buffer (column
    major with leading dimension ld); C0(:,ist) copies NGWX entries from
    column ist, so with ld < NGWX it reads into the next column exactly as
    the reference does.  The scatter runs over ig < NGW_ik, dropping the last
    plane wave (:117).  Returns (rhoe_increment, ekin_increment, C0)."""
    nr = cell["nr"]
    nnr = nr[0] * nr[1] * nr[2]
    rho = np.zeros(nnr)
    c0 = np.zeros((ngwx, nx), dtype=complex)
    idx = cell["n123"][: ngw - 1].astype(np.int64) - 1
    xkin = 0.0
    for ist in range(nx):
        wdotf = wkpt * focc[ist]
        c0[:, ist] = eigvec_flat[ist * ld: ist * ld + ngwx]
        ct = c0[: ngw - 1, ist]
        scg = np.abs(ct) ** 2
        ss = float(np.sum(scg))
        if abs(ss - 1.0) > 6.0e-3:
            raise RuntimeError(f"Wrong charge density in G-space: {ss} (state {ist + 1})")
        xkin += float(np.sum(cell["xkg"][: ngw - 1] * scg)) * wdotf * 0.5
        c = np.zeros(nnr, dtype=complex)
        c[idx] = ct
        c = fft_inverse(c, nr)
        rho += np.abs(c) ** 2 * (wdotf / omega)
    return rho, xkin * cell["tpiba2"], c0


def eval_enl(cell, c0, ngw, nx, focc, wkpt):
    """EvalENL.cpp:5-49: FNL = C0^T (PKG_A conj(EIGR)) (unconjugated C0),
    ENL = sum w f |FNL|^2 WNL.  Returns (ENL, FNL[nx, nproj])."""
    beta, w = projectors(cell, ngw)
    fnl = c0[:ngw, :nx].T @ beta.conj()
    enl = float(np.sum(wkpt * (focc[:nx, None] * np.abs(fnl) ** 2) * w[None, :]))
    return enl, fnl


# ---------------------------------------------------------------- SCF pieces
# Restatements of the steps around the eigensolver; the engine's versions are
# in ffr-pspw-dft-c_b200/csrc/scf.cu.

def _pz_point(r):
    """xc_PZ.cpp:24-59 at one point: (ux + uc, ex + ec); zeros for r <= 1e-13."""
    A, B, C = -0.1423, 1.0529, 0.3334
    a, b, c, d = 0.0311, -0.0480, 0.0020, -0.0116
    if r <= 1.e-13:
        return 0.0, 0.0
    ax = -(3.0 / 4.0) * (3.0 / 2.0 / np.pi) ** (2.0 / 3.0)
    rs = (3.0 / (4.0 * np.pi * r)) ** (1.0 / 3.0)
    rrs = np.sqrt(rs)
    ex = ax / rs
    ux = 4.0 / 3.0 * ex
    if rs >= 1.0:
        bpr = 1.0 + B * rrs + C * rs
        ec = A / bpr
        uc = (1.0 + 7.0 / 6.0 * B * rrs + 4.0 / 3.0 * C * rs) * ec / bpr
    else:
        rsl = np.log(rs)
        ec = a * rsl + b + c * rs * rsl + d * rs
        uc = (2.0 * d - c) / 3.0 * rs + b - a / 3.0 + a * rsl + 2.0 * c / 3.0 * rs * rsl
    return ux + uc, ex + ec


def xc_pz(rho):
    """xc_PZ.cpp:7-63: (vxc, Exc = sum rho (ex + ec)).  A point with rho < -0.1
    keeps the previous point's values (the loop variables are not reset)."""
    vxc = np.zeros(len(rho))
    exc = 0.0
    v = e = 0.0
    for i, r in enumerate(rho):
        if not r < -0.1:
            v, e = _pz_point(float(r))
        vxc[i] = v
        exc = exc + r * e
    return vxc, exc


def normalize_rho(rho, omega, nel):
    """NormalizeRho.cpp:7-33 (negatives clipped, scaled to NEL electrons)."""
    r = np.array(rho, dtype=float, copy=True)
    r[r < 0.0] = 0.0
    s = r.sum()
    if s < 1.0e-15:
        raise RuntimeError("NormalizeRho: sum(rho) too small")
    truesum = len(r) * nel / omega
    return r * truesum / s


def kerker_prec(x, cell, beta, q0):
    """KerkerRhoMix.cpp:53-81: filter the wavefunction-sphere components of
    FFT(x) by beta gg/(gg+q0); the others are unchanged."""
    c = fft_forward(np.asarray(x, dtype=complex), cell["nr"])
    ngw = int(cell["ngw"])
    idx = np.asarray(cell["n123"])[:ngw].astype(np.int64) - 1
    gg = np.asarray(cell["xkg"])[:ngw]
    c[idx] = (beta * gg / (gg + q0)) * c[idx]
    return fft_inverse(c, cell["nr"]).real


def eval_energy(rho, local, cell, ekin, enl):
    """EvalEnergy.cpp:5-163.  local: dict with gidx (0-based grid index of the
    density G's, G = 0 first), g (|G|^2, tpiba^2 units), vp and rp (sums over
    species of SFAC*VPS and SFAC*RHOPS), omega, esr, eself.  Returns (V_eff,
    energies).  Grid points outside the density sphere keep FFT(rho)."""
    nr = cell["nr"]
    c = fft_forward(np.asarray(rho, dtype=complex), nr)
    gidx, g, vp, rp = local["gidx"], local["g"], local["vp"], local["rp"]
    eps = vp[0] * np.conj(c[0])
    rhet = c[gidx[1:]]
    rhog = rhet + rp[1:]
    fpibg = 4.0 * np.pi / (cell["tpiba2"] * g[1:])
    vcg = fpibg * rhog
    eh = np.sum(0.5 * vcg * np.conj(rhog))
    eps = eps + np.sum(np.conj(rhet) * vp[1:])
    vtemp = np.concatenate([[vp[0]], vcg + vp[1:]])
    # scatter in G order (EvalEnergy.cpp:117-119): on a grid smaller than the
    # density sphere needs, G alias onto one point and the last one stays
    c[gidx] = vtemp
    last = len(gidx) - 1 - np.unique(np.asarray(gidx)[::-1], return_index=True)[1]
    c[np.asarray(gidx)[last]] = vtemp[last]
    v = fft_inverse(c, nr)
    vxc, exc = xc_pz(rho)
    veff = v.real + vxc
    n = len(rho)
    EXC = exc * local["omega"] / n
    EHT = eh.real * local["omega"] + local["esr"] - local["eself"]
    EPSEU = eps.real * local["omega"]
    return veff, dict(ETOT=ekin + EHT + EPSEU + enl + EXC, EKIN=ekin, EHT=EHT, EPSEU=EPSEU,
                      ENL=enl, EXC=EXC)


class Mixer:
    """SimpleRhoMix.cpp, KerkerRhoMix.cpp:5-50, AndersonRhoMix.cpp:8-91,
    PulayRhoMix.cpp:5-91 and BroydenRhoMix.cpp:10-104 with their history
    (zero at the start, as the ChebySCF loop allocates it).  kind: 0 simple,
    1 Kerker, 2 Anderson, 3 Pulay, 4 Broyden (alpha = beta, w0 = 0.01)."""

    def __init__(self, kind, nnr, cell, mixdim=0, beta=0.25, q0=0.0, omega=1.0, nel=0.0,
                 rho_old=None):
        self.kind, self.cell, self.mixdim, self.beta, self.q0 = kind, cell, mixdim, beta, q0
        self.omega, self.nel = omega, nel
        ncol = mixdim if kind == 3 else (3 if kind == 2 else (2 if kind == 4 else 1))
        self.h = np.zeros((nnr, ncol))
        self.f = np.zeros((nnr, ncol))
        self.g = np.zeros((nnr, 2))
        if kind == 4:
            self.df = np.zeros((nnr, mixdim))
            self.u = np.zeros((nnr, mixdim))
            self.a = np.zeros((mixdim, mixdim))
        if rho_old is not None:
            self.h[:, 0] = rho_old

    def _broyden(self, it, rho):
        alpha, w0, md, n = self.beta, 0.01, self.mixdim, len(rho)
        h, f, df, u, a = self.h, self.f, self.df, self.u, self.a
        m = min(it + 1, md)
        jc, kp, kc = it % m, (it - 1) % 2, it % 2
        f[:, kc] = rho - h[:, kp]
        d = np.sqrt(float(f[:, kc] @ f[:, kc]) / n)
        df[:, jc] = f[:, kc] - f[:, kp]
        t1 = np.sqrt(float(df[:, jc] @ df[:, jc]))
        if t1 > 1.e-8:
            t1 = 1.0 / t1
        df[:, jc] = t1 * df[:, jc]
        u[:, jc] = alpha * df[:, jc] + t1 * (h[:, kp] - h[:, kc])
        c = np.array([df[:, k] @ f[:, kc] for k in range(m)])
        for k in range(m):
            a[k, jc] = a[jc, k] = df[:, jc] @ df[:, k]
        beta = a[:m, :m] + w0 * w0 * np.eye(m)
        gamma = c @ np.linalg.inv(beta)
        rho = h[:, kp] + alpha * f[:, kc] - u[:, :m] @ gamma
        h[:, kc] = rho
        return rho, d

    def mix(self, it, rhoe):
        rhoe = np.array(rhoe, dtype=float, copy=True)
        b, h, f, g, n = self.beta, self.h, self.f, self.g, len(rhoe)
        if self.kind == 0:
            d = np.sum((rhoe - h[:, 0]) ** 2)
            rhoe = b * rhoe + (1.0 - b) * h[:, 0]
            h[:, 0] = rhoe
            return rhoe, np.sqrt(d / n)
        if self.kind == 1:
            d = np.sum((rhoe - h[:, 0]) ** 2)
            rhoe = h[:, 0] + kerker_prec(rhoe - h[:, 0], self.cell, b, self.q0)
            h[:, 0] = rhoe
            return rhoe, np.sqrt(d / n)
        if self.kind == 2:
            if it == 1:
                h[:, 0] = rhoe
                f[:, 0] = 0.0
                return rhoe, 1.0
            j0, j1, j2 = (it - 1) % 3, (it - 2) % 3, (it - 3) % 3
            f[:, j0] = rhoe - h[:, j1]
            d = float(f[:, j0] @ f[:, j0])
            if it == 2:
                rhoe = b * rhoe + (1.0 - b) * h[:, j1]
                h[:, j0] = rhoe
                return rhoe, d
            g[:, 0] = f[:, j1] - f[:, j0]
            d11 = g[:, 0] @ g[:, 0]
            r1 = f[:, j0] @ g[:, 0]
            if it == 3:
                t1 = -r1 / d11
                rhoe = (1 - t1) * h[:, j1] + t1 * h[:, j2] + b * (f[:, j0] + t1 * g[:, 0])
            else:
                g[:, 1] = f[:, j2] - f[:, j0]
                d22 = g[:, 1] @ g[:, 1]
                d12 = g[:, 0] @ g[:, 1]
                r2 = f[:, j0] @ g[:, 1]
                t1 = d11 * d22
                t2 = t1 - d12 * d12
                if abs(t2) > abs(t1) * 1.0e-8:
                    t1, t2 = (-r1 * d22 + r2 * d12) / t2, (r1 * d12 - r2 * d11) / t2
                else:
                    t1 = t2 = 0.0
                rhoe = ((1 - t1 - t2) * h[:, j1] + t1 * h[:, j2] + t2 * h[:, j0]
                        + b * (f[:, j0] + t1 * g[:, 0] + t2 * g[:, 0]))
            h[:, j0] = rhoe
            return rhoe, d
        if self.kind == 4:
            return self._broyden(it, rhoe)
        # Pulay
        md = self.mixdim
        if it < md:
            rhoe = b * rhoe + (1.0 - b) * h[:, it - 1]
            f[:, it] = kerker_prec(rhoe - h[:, it - 1], self.cell, 1.0, self.q0)
            h[:, it] = rhoe
            return rhoe, np.sqrt(np.sum(f[:, it] ** 2) / n)
        jc, jn = it % md, (it + 1) % md
        m = min(it + 1, md) + 1
        f[:, jc] = kerker_prec(rhoe - h[:, jc], self.cell, 1.0, self.q0)
        d = np.sqrt(np.sum(f[:, jc] ** 2) / n)
        a = np.zeros((m, m))
        for i in range(m - 1):
            for j in range(i, m - 1):
                a[i, j] = f[:, i] @ f[:, j]
                a[j, i] = a[i, j]
            a[i, m - 1] = a[m - 1, i] = 1.0
        rhs = np.zeros(m)
        rhs[m - 1] = 1.0
        alpha = np.linalg.solve(a, rhs)
        rhoe = sum(alpha[j] * (h[:, j] + f[:, j]) for j in range(m - 1))
        rhoe = normalize_rho(rhoe, self.omega, self.nel)
        h[:, jn] = rhoe
        return rhoe, d
