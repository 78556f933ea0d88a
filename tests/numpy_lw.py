"""A second, independent restatement of the TreeMesh LW rhs in vectorised numpy (test helper).

It follows the reference stage by stage but is written in array form (all elements and nodes at once),
so that a transcription slip in the C++ oracle's loop form would show up as a disagreement. Supports
LW depth 3 (N=3, src/solvers/dgsem_tree/dg_2d.jl:674-916) and depth 4 (N>=4, :918-1267), periodic
meshes, Rusanov flux with max_abs_speed_naive in TreeMesh argument order (:1928), weak-form surface
integral and apply_jacobian (Trixi).
"""
import numpy as np


def euler_fluxes(u, gamma=1.4):
    rho, m1, m2, e = u[..., 0], u[..., 1], u[..., 2], u[..., 3]
    v1, v2 = m1 / rho, m2 / rho
    p = (gamma - 1) * (e - 0.5 * (m1 * v1 + m2 * v2))
    f = np.stack([m1, m1 * v1 + p, m1 * v2, (e + p) * v1], axis=-1)
    g = np.stack([m2, m2 * v1, m2 * v2 + p, (e + p) * v2], axis=-1)
    return f, g


def speed_naive(ul, ur, orientation, gamma=1.4):
    def prim(u):
        rho = u[..., 0]
        v1, v2 = u[..., 1] / rho, u[..., 2] / rho
        p = (gamma - 1) * (u[..., 3] - 0.5 * (u[..., 1] * v1 + u[..., 2] * v2))
        return rho, v1, v2, p
    rl, v1l, v2l, pl = prim(ul)
    rr, v1r, v2r, pr = prim(ur)
    vl, vr = (v1l, v1r) if orientation == 1 else (v2l, v2r)
    cl, cr = np.sqrt(gamma * pl / rl), np.sqrt(gamma * pr / rr)
    return np.maximum(np.abs(vl), np.abs(vr)) + np.maximum(cl, cr)


def rhs(u, mesh, D, Dhat, w, dt, gamma=1.4):
    """u: [E, j, i, v] (reference u[v,i,j,e]); returns du with the same layout, plus U, F(x), G(y)."""
    E, n, _, _ = u.shape
    N = n - 1
    ij = mesh.inverse_jacobian[:, None, None, None]

    def contract(fx, gy):
        # sum_k D[i,k] fx[e, j, k] + sum_k D[j,k] gy[e, k, i]
        return np.einsum("ik,ejkv->ejiv", D, fx) + np.einsum("jk,ekiv->ejiv", D, gy)

    f0, g0 = euler_fluxes(u, gamma)
    F, G, U = f0.copy(), g0.copy(), u.copy()
    ut = -dt * contract(f0, g0) * ij
    U += 0.5 * ut
    up, um, upp, umm = u + ut, u - ut, u + 2 * ut, u - 2 * ut
    fl = lambda s: euler_fluxes(s, gamma)
    (fpp, gpp), (fp, gp), (fm, gm), (fmm, gmm) = fl(upp), fl(up), fl(um), fl(umm)
    ft = (-fpp + 8 * fp - 8 * fm + fmm) / 12.0
    gt = (-gpp + 8 * gp - 8 * gm + gmm) / 12.0
    F += 0.5 * ft
    G += 0.5 * gt
    utt = -dt * contract(ft, gt) * ij
    U += utt / 6.0
    up += 0.5 * utt
    um += 0.5 * utt
    upp += 2 * utt
    umm += 2 * utt
    if N >= 4:
        (fpp, gpp), (fp, gp), (fm, gm), (fmm, gmm) = fl(upp), fl(up), fl(um), fl(umm)
        ftt = (-fpp + 16 * fp - 30 * f0 + 16 * fm - fmm) / 12.0
        gtt = (-gpp + 16 * gp - 30 * g0 + 16 * gm - gmm) / 12.0
    else:
        (fp, gp), (fm, gm) = fl(up), fl(um)
        ftt = fp - 2 * f0 + fm
        gtt = gp - 2 * g0 + gm
    F += ftt / 6.0
    G += gtt / 6.0
    uttt = -dt * contract(ftt, gtt) * ij
    U += uttt / 24.0
    um += -uttt / 6.0
    up += uttt / 6.0
    umm += -4.0 / 3.0 * uttt
    upp += 4.0 / 3.0 * uttt
    (fpp, gpp), (fp, gp), (fm, gm), (fmm, gmm) = fl(upp), fl(up), fl(um), fl(umm)
    fttt = 0.5 * (fpp - 2 * fp + 2 * fm - fmm)
    gttt = 0.5 * (gpp - 2 * gp + 2 * gm - gmm)
    F += fttt / 24.0
    G += gttt / 24.0
    if N >= 4:
        utttt = -dt * contract(fttt, gttt) * ij
        U += utttt / 120.0
        um += utttt / 24.0
        up += utttt / 24.0
        umm += 2.0 / 3.0 * utttt
        upp += 2.0 / 3.0 * utttt
        (fpp, gpp), (fp, gp), (fm, gm), (fmm, gmm) = fl(upp), fl(up), fl(um), fl(umm)
        F += 0.5 * (fpp - 4 * fp + 6 * f0 - 4 * fm + fmm) / 120.0
        G += 0.5 * (gpp - 4 * gp + 6 * g0 - 4 * gm + gmm) / 120.0
    du = contract_hat = np.einsum("ik,ejkv->ejiv", Dhat, F) + np.einsum("jk,ekiv->ejiv", Dhat, G)
    # interfaces (periodic TreeMesh): Fn = 1/2 (F_L + F_R) - 1/2 lambda(U_L, U_R) (u_R - u_L)
    sfv = np.zeros((E, 4, n, 4))   # [e, face, l, v]
    ids = mesh.interface_neighbor_ids - 1
    for (le, re), o in zip(ids, mesh.interface_orientations):
        if o == 1:
            uL, uR, UL, UR, FL, FR = u[le, :, n - 1], u[re, :, 0], U[le, :, n - 1], U[re, :, 0], F[le, :, n - 1], F[re, :, 0]
            fL, fR = 1, 0
        else:
            uL, uR, UL, UR, FL, FR = u[le, n - 1, :], u[re, 0, :], U[le, n - 1, :], U[re, 0, :], G[le, n - 1, :], G[re, 0, :]
            fL, fR = 3, 2
        lam = speed_naive(UL, UR, o, gamma)[:, None]
        Fn = 0.5 * (FL + FR) - 0.5 * lam * (uR - uL)
        sfv[le, fL] = Fn
        sfv[re, fR] = Fn
    du[:, :, 0] -= sfv[:, 0] / w[0]
    du[:, :, n - 1] += sfv[:, 1] / w[n - 1]
    du[:, 0, :] -= sfv[:, 2] / w[0]
    du[:, n - 1, :] += sfv[:, 3] / w[n - 1]
    du *= -ij
    del contract_hat
    return du, U, F, G
