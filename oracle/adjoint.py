"""Vector-Jacobian products of the PM force and of the P(k) loss (float64 numpy).

The reference has no adjoint: these restate the transposes of the operators in
`native/DiscoDJNative/src/nbody/pm.jl` (scatter pm.jl:57-74, Kφ pm.jl:389-391, FD
gradient pm.jl:330-342, gather pm.jl:344-364, shift average pm.jl:513-519) and of
`evaluate_power_spectrum` (analysis/power_spectrum.jl:25-79). The CIC adjoint gather
follows the pattern of `_cic_gather_kernel!` (src/field/sheet_deposit.jl:75-94): the
weight derivative of every node times the mesh cotangent. They are checked against
central finite differences of the float64 forward restatements in the tests.
Test infrastructure only (see `oracle/__init__.py`).
"""
from __future__ import annotations

import numpy as np

from . import pm as opm
from .pm import irfftn, rfftn


def dwk(W: int, d):
    """d/dd of wk(W, |d|) for the signed distance d = g − node (pm.jl:49-51 differentiated)."""
    d = np.asarray(d, dtype=np.float64)
    a = np.abs(d)
    s = np.sign(d)
    if W == 2:
        return np.where(a > 1, 0.0, -s)
    if W == 3:
        return np.where(a > 1.5, 0.0, np.where(a > 0.5, -(1.5 - a) * s, -2.0 * d))
    if W == 4:
        return np.where(a > 2, 0.0, np.where(a > 1, -0.5 * (2 - a) ** 2 * s, -2.0 * d + 1.5 * d * a))
    raise ValueError("worder must be 2, 3 or 4")


def _stencil(X, res, L, W):
    """Per axis: node indices, weights and weight derivatives (d/dX) of the W nodes."""
    g = opm._grid_coords(X, res, L)
    out = []
    for a in range(3):
        b = opm.wbase(W, g[a])
        nodes, ws, ds = [], [], []
        for o in opm.woffsets(W):
            d = g[a] - (b + o)
            nodes.append(np.mod(b + o, res))
            ws.append(opm.wk(W, np.abs(d)))
            ds.append(dwk(W, d) * (res / L))
        out.append((nodes, ws, ds))
    return out


def gather_grad(fields, X, res, L, W):
    """J[p, a, c] = Σ_n ∂W(X_p − n)/∂X_a · fields[c][n] for a list of meshes."""
    st = _stencil(X, res, L, W)
    J = np.zeros((X.shape[0], 3, len(fields)))
    (nx, wx, dx), (ny, wy, dy), (nz, wz, dz) = st
    for iz in range(W):
        for iy in range(W):
            for ix in range(W):
                grads = (dx[ix] * wy[iy] * wz[iz], wx[ix] * dy[iy] * wz[iz], wx[ix] * wy[iy] * dz[iz])
                for c, f in enumerate(fields):
                    v = f[nx[ix], ny[iy], nz[iz]]
                    for a in range(3):
                        J[:, a, c] += grads[a] * v
    return J


def scatter_weighted(X, weights, res, L, W):
    """mesh[n] += weights_p · W(X_p − n) (pm_scatter with per-particle masses)."""
    st = _stencil(X, res, L, W)
    (nx, wx, _), (ny, wy, _), (nz, wz, _) = st
    flat = np.zeros(res ** 3)
    for iz in range(W):
        for iy in range(W):
            for ix in range(W):
                idx = (nx[ix] * res + ny[iy]) * res + nz[iz]
                flat += np.bincount(idx, weights=weights * wx[ix] * wy[iy] * wz[iz], minlength=res ** 3)
    return flat.reshape(res, res, res)


def fd_apply(f, c_axis, coef):
    """(D_c f)(n) = Σ_t c_t (f(n + t e_c) − f(n − t e_c)) (pm.jl:330-342 without the sign)."""
    out = np.zeros_like(f)
    for t, ct in enumerate(coef, start=1):
        if ct != 0.0:
            out += ct * (np.roll(f, -t, axis=c_axis) - np.roll(f, t, axis=c_axis))
    return out


def _poisson(cfg, mesh):
    """φ = K ∗ mesh: the unnormalised brfft of Kφ·rfft(mesh) (pm.jl:494-495); symmetric."""
    res = cfg.res_pm
    return irfftn(rfftn(mesh) * opm.k_phi(cfg), res) * res ** 3


def _positions(cfg, psi):
    n, L = cfg.n_part, cfg.boxsize
    q1 = opm._lagr1d(n, L)
    X = np.empty_like(psi, dtype=np.float64)
    X[..., 0] = psi[..., 0] + q1[:, None, None]
    X[..., 1] = psi[..., 1] + q1[None, :, None]
    X[..., 2] = psi[..., 2] + q1[None, None, :]
    return X


def pm_acceleration_fd(cfg, psi):
    """The PM force with the real-space FD gradient (the form the CUDA library uses)."""
    n, res, L, W = cfg.n_part, cfg.res_pm, cfg.boxsize, cfg.worder
    coef = opm.fd_coeffs(cfg.grad_order, L / res)
    X = _positions(cfg, psi)
    shifts = opm.aa_shifts(cfg.antialias, 0.5 * L / res)
    acc = np.zeros((n ** 3, 3))
    for s in shifts:
        Xs = (X + np.asarray(s)[None, None, None, :]).reshape(-1, 3)
        phi = _poisson(cfg, opm.pm_scatter(np.zeros((res, res, res)), Xs, res, L, W))
        for c in range(3):
            acc[:, c] += opm.pm_gather(-fd_apply(phi, c, coef), Xs, res, L, W)
    acc /= len(shifts)
    return acc.reshape(n, n, n, 3)


def pm_acceleration_vjp(cfg, psi, acc_bar):
    """Ψ̄ = (∂acc/∂Ψ)ᵀ ā for finite-difference gradients (orders 2/4/6), n_resample = 1.

    Per shift s (acc = mean over shifts): acc_c = Σ_n W G_c with G_c = −D_c φ,
    φ = K ∗ ρ, ρ = Σ_p W. Then
      Ψ̄_a += Σ_c ā_c Σ_n ∂_a W · G_c               (the interpolation weights)
      Ḡ_c = Σ_p ā_c W,  φ̄ = Σ_c D_c Ḡ_c (Dᵀ = −D),  ρ̄ = K ∗ φ̄ (K symmetric)
      Ψ̄_a += Σ_n ∂_a W · ρ̄                        (the deposit weights)."""
    if cfg.grad_order == 0 or cfg.n_resample > 1:
        raise ValueError("the VJP covers finite-difference gradients without resampling")
    n, res, L, W = cfg.n_part, cfg.res_pm, cfg.boxsize, cfg.worder
    coef = opm.fd_coeffs(cfg.grad_order, L / res)
    X = _positions(cfg, psi)
    ab = np.asarray(acc_bar, dtype=np.float64).reshape(-1, 3)
    shifts = opm.aa_shifts(cfg.antialias, 0.5 * L / res)
    ns = len(shifts)
    out = np.zeros((n ** 3, 3))
    for s in shifts:
        Xs = (X + np.asarray(s)[None, None, None, :]).reshape(-1, 3)
        phi = _poisson(cfg, opm.pm_scatter(np.zeros((res, res, res)), Xs, res, L, W))
        G = [-fd_apply(phi, c, coef) for c in range(3)]
        J = gather_grad(G, Xs, res, L, W)                       # (N, 3 positions, 3 components)
        out += np.einsum("pac,pc->pa", J, ab) / ns
        phibar = np.zeros((res, res, res))
        for c in range(3):
            phibar += fd_apply(scatter_weighted(Xs, ab[:, c] / ns, res, L, W), c, coef)
        rhobar = _poisson(cfg, phibar)
        out += gather_grad([rhobar], Xs, res, L, W)[:, :, 0]
    return out.reshape(n, n, n, 3)


def power_spectrum_vjp(cfg_res, n_part, boxsize, psi, pk_bar, bins=32, logarithmic=True):
    """Ψ̄ of a loss through P(k) of the CIC density of X = q + Ψ (bins as
    `evaluate_power_spectrum`, δ = mesh·res³/n³ − 1), given ∂loss/∂P_b.

    P_b = (V/res⁶)·Σ_{k∈b} |δ̂_k|² / N_b over the full spectrum (the half-spectrum
    weights 0.5 on the self-conjugate planes count those modes once), so
    ∂loss/∂δ(n) = Σ_b P̄_b·(2V/res⁶/N_b)·Σ_{k∈b} δ̂_k e^{ik·n}: an unnormalised C2R of
    the binned, scaled spectrum."""
    import math

    from .power import bin_edges
    res, L = cfg_res, boxsize
    cfg = opm.PMConfig(res_pm=res, n_part=n_part, boxsize=L, worder=2)
    X = _positions(cfg, psi).reshape(-1, 3)
    mesh = opm.pm_scatter(np.zeros((res, res, res)), X, res, L, 2)
    f = rfftn(mesh * (res ** 3 / n_part ** 3))
    dk = 2 * math.pi / L
    kfull = np.array([i if i <= res // 2 else i - res for i in range(res)]) * dk
    khalf = np.arange(res // 2 + 1) * dk
    k_arr = np.sqrt(kfull[:, None, None] ** 2 + kfull[None, :, None] ** 2 + khalf[None, None, :] ** 2)
    edges = bin_edges(res, L, bins, logarithmic)
    w = np.ones_like(k_arr)
    w[:, :, 0] = 0.5
    w[:, :, -1] = 0.5
    V = L ** 3
    H = np.zeros_like(f)
    for b in range(bins):
        mask = (k_arr >= edges[b]) & (k_arr < edges[b + 1])
        wsum = w[mask].sum()
        if wsum == 0:
            continue
        # P_b = (V/res⁶) Σ_half w|δ̂|² / Σ_half w; d/dδ̂ of Σ_half w|δ̂|² over the
        # half spectrum maps to the full-spectrum form below (Σ_half w = N_b/2)
        H[mask] = pk_bar[b] * (V / res ** 6) / wsum * f[mask]
    dbar = irfftn(H, res) * res ** 3                      # Σ_full H_k e^{ik·n}
    mbar = dbar * (res ** 3 / n_part ** 3)
    return gather_grad([mbar], X, res, L, 2)[:, :, 0].reshape(n_part, n_part, n_part, 3)
