"""Oracle restatement of ``rqutils/ground_locg.py`` (test infrastructure only).

``ground_locg`` follows ground_locg.py:128-162 and ``_ground_locg_callable`` :188-423 (debug
diagnostics omitted), ``_project_out`` :426-464, ``eigenpair_2x2`` :467-478 and
``eigenpair_3x3`` :481-514.  NumPy FP64; XLA's reduction order is not reproduced (parity
unpinned at that boundary, tolerances used).
"""
import numpy as np


def _norm(v):
    return np.sqrt(np.sum((v.conjugate() * v).real))


def _dot(a, b):
    return np.sum(a.conjugate() * b)


def project_out(basis, vector, normalize=True, rounds=2):
    """ground_locg.py:426-464."""
    vector = vector.copy()
    for iround in range(2 * rounds):
        ips = [_dot(vb, vector) for vb in basis]
        for vb, ip in zip(basis, ips):
            vector = vector - vb * ip
        if normalize and iround < rounds:
            norm = _norm(vector)
            vector = vector / (1. if norm == 0. else norm)
    if normalize:
        vector = vector * np.asarray(_norm(vector) >= 0.99).astype(vector.dtype)
    return vector


def eigenpair_2x2(mat):
    """ground_locg.py:467-478."""
    d = np.diagonal(mat).real
    det = d[0] * d[1] - np.abs(mat[1, 0]) ** 2
    tr = d[0] + d[1]
    eigval = (tr - np.sqrt(tr * tr - 4. * det)) * 0.5
    eigvec = np.array([(d[1] - eigval + np.conjugate(mat[1, 0])) / (d[0] - eigval + mat[1, 0]),
                       -1.], dtype=mat.dtype)
    e0 = eigvec[0]
    eigvec = eigvec / np.sqrt(e0.real * e0.real + e0.imag * e0.imag + 1.)
    return eigval, eigvec


def eigenpair_3x3(mat):
    """ground_locg.py:481-514: Cardano's method after J. Kopp, Int. J. Mod. Phys. C 19, 523
    (2008)."""
    d = np.diagonal(mat).real
    modod = np.abs(mat[[1, 2, 2], [0, 0, 1]]) ** 2
    c2 = -np.sum(d)
    c1 = np.sum(d * np.roll(d, 1)) - np.sum(modod)
    c0 = np.sum(d * modod[::-1])
    c0 -= np.prod(d)
    c0 -= 2. * (mat[0, 2] * mat[1, 0] * mat[2, 1]).real
    p = c2 * c2 - 3. * c1
    q = -13.5 * c0 - c2 * c2 * c2 + 4.5 * c2 * c1
    phi = np.arctan2(np.sqrt(27. * (0.25 * c1 * c1 * (p - c1) + c0 * (q + 6.75 * c0))), q) / 3.
    cphi = np.cos(phi)
    sphi = np.sin(phi)
    xmin = min(2. * cphi, -cphi - np.sqrt(3.) * sphi, -cphi + np.sqrt(3.) * sphi)
    eigval = np.sqrt(p) / 3. * xmin - c2 / 3.
    v0 = mat[:, 1].copy()
    v0[1] -= eigval
    v1 = mat[:, 2].copy()
    v1[2] -= eigval
    eigvec = np.cross(v0, v1).conjugate()
    re, im = eigvec.real, eigvec.imag
    eigvec = eigvec / np.sqrt(np.sum(re * re) + np.sum(im * im))
    return eigval, eigvec


def ground_locg(mat, xinit, args=(), orth=(), maxiter=1000, tol=None, vspace=None,
                return_history=False):
    """Restates ``ground_locg`` + ``_ground_locg_callable`` (ground_locg.py:128-423).

    ``mat`` is a callable ``mat(x, *args)`` or a dense matrix.  Returns (eigval, eigvec, niter)
    and, if ``return_history``, the list of residual norms per body iteration.
    """
    if not isinstance(orth, tuple):
        orth = (orth,)
    if not callable(mat):
        dense = np.asarray(mat)
        if isinstance(xinit, (int, np.integer)):
            vspace = (dense.shape[1], dense.dtype)

        def matvec(x):
            return dense @ x
        args = ()
    else:
        def matvec(x):
            return mat(x, *args)

    orth = tuple(v / _norm(v) for v in orth)                       # :208
    if isinstance(xinit, (int, np.integer)):                       # :210-222
        ndim, dtype = vspace[:2]
        xinit = (np.arange(ndim) == xinit).astype(dtype)
        if orth:
            xinit = project_out(orth, xinit)
    xinit = np.asarray(xinit)
    if tol is None:                                                # :224-225
        tol = float(np.finfo(xinit.dtype).eps)

    def compute_sas(*vectors):                                     # :251-264
        nv = len(vectors)
        sas = np.zeros((nv, nv), dtype=vectors[0].dtype)
        mvs = []
        for iv1, v1 in enumerate(vectors):
            mv1 = matvec(v1)
            mvs.append(mv1)
            for iv2 in range(iv1 + 1, nv):
                sas[iv2, iv1] = _dot(vectors[iv2], mv1)
        sas = sas + sas.conjugate().T
        for iv1, (v1, mv1) in enumerate(zip(vectors, mvs)):
            sas[iv1, iv1] = _dot(v1, mv1)
        return sas

    def rayleigh_ritz(*vectors):                                   # :266-271
        sas = compute_sas(*vectors)
        if len(vectors) == 2:
            return eigenpair_2x2(sas)
        return eigenpair_3x3(sas)

    xcurr = xinit / _norm(xinit)                                   # :388
    # body_iter0 (:280-291)
    ax = matvec(xcurr)
    if orth:
        ax = project_out(orth, ax, normalize=False)
    theta = _dot(xcurr, ax).real
    rcurr = ax - theta * xcurr
    # body_iter1 (:293-322)
    norm_r = _norm(rcurr)
    if norm_r == 0.:
        ycurr = np.zeros_like(xcurr)
    else:
        tmp_p = rcurr / norm_r
        theta, kappa = rayleigh_ritz(xcurr, tmp_p)
        tmp_t = tmp_p * kappa[0] - xcurr * kappa[1]
        tmp_u = xcurr * kappa[0] + tmp_p * kappa[1]
        xnext = tmp_u / _norm(tmp_u)
        ycurr = tmp_t / _norm(tmp_t)
        if orth:
            xnext = project_out(orth, xnext)
        rcurr = matvec(xnext) - theta * xnext
        if orth:
            rcurr = project_out(orth, rcurr, normalize=False)
        xcurr = xnext

    niter = 0
    converged = False
    history = []
    while niter < maxiter and not converged:                       # :412-416
        tmp_p = project_out((xcurr, ycurr), rcurr)                 # body (:324-383)
        theta, kappa = rayleigh_ritz(xcurr, ycurr, tmp_p)
        tmp_s = ycurr * kappa[1] + tmp_p * kappa[2]
        norm_s = _norm(tmp_s)
        tmp_t = tmp_s * (kappa[0] / norm_s) - xcurr * norm_s
        tmp_u = xcurr * kappa[0] + tmp_s
        xnext = tmp_u / _norm(tmp_u)
        ynext = tmp_t / _norm(tmp_t)
        if orth:
            xnext = project_out(orth, xnext)
        axnext = matvec(xnext)
        rnext = axnext - xnext * theta
        if orth:
            rnext = project_out(orth, rnext, normalize=False)
        reltol = (_norm(axnext) - theta) * xcurr.shape[0] * 10
        norm_rnext = _norm(rnext)
        converged = bool(norm_rnext < tol * reltol)
        history.append(norm_rnext)
        xcurr, ycurr, rcurr = xnext, ynext, rnext
        niter += 1

    if return_history:
        return theta, xcurr, niter, history
    return theta, xcurr, niter
