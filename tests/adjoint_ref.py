"""CPU restatement of the adjoint of the direct UW12 terms (test infrastructure).

libuw12 has no adjoint; this numpy version of the reverse sweep that the CUDA
path implements is the checker for it, and is itself checked against central
finite differences of the oracle energy (tests/test_adjoint_math.py).

Energy of the direct terms (``form_fock(..., indirect_term=False)``), summed
over spin pairs with the spin factor f(s, s'):
    E2 = 1/2 f X_D[s] . (L_WV X_D[s'])          (two_electron.cpp:37-81)
    E4 = 1/2 f < t~[s'], t[s] >                  (four_electron.cpp:80-137)
    E3 = -f < X[s], t~[s'] >                     (direct_utils.cpp:136-157)
with t = B2_W^T B2_V, t~ = L_W t L_V, X = Wst_W^T (I (x) S^-1) Wst_V in the
metric eigenbasis.  In the original aux basis these depend on the metrics
only through K = J2^-1, so dE/dJ2 = -K G K with G = dE/dK, which in the
eigenbasis is a product of the M x M intermediates (no eigenvector
derivatives); dE/dJ3 follows the transforms backwards with P2 fixed.
"""
from __future__ import annotations

import numpy as np

from oracle import uw12_oracle as O


def spin_factor(ns, s, sp, s_os, s_ss):
    return O.get_energy_spin_factor(ns, s, sp, s_os, s_ss)


def direct_energy(W, V, WV, abs_p, orbitals, occ, n_active, s_os, s_ss):
    """Energy of the direct terms through the oracle."""
    return O.form_fock(W, V, WV, abs_p, orbitals, occ, n_active, False, False, s_os,
                       s_ss).energy


def _pack_sym_sum(G):
    """Gradient on the packed lower triangle of a symmetric matrix: G[i,j] + G[j,i]
    off the diagonal, G[i,i] on it; packed row i(i+1)/2 + j, j <= i."""
    n = G.shape[0]
    out = np.zeros(n * (n + 1) // 2)
    for i in range(n):
        for j in range(i + 1):
            out[i * (i + 1) // 2 + j] = G[i, j] + (G[j, i] if i != j else 0.0)
    return out


def direct_adjoint(Wb, Vb, WVb, abs_p, orbitals, occ, n_active, s_os, s_ss):
    """dE/d(J3_0, J3_ri_0, J2) of W, V and dE/d(J3_0, J2) of WV for the direct terms."""
    ns = len(orbitals)
    Co = O.occupation_weighted_orbitals(orbitals, occ)
    Ca = O.freeze_core(Co, n_active)
    W = O.Integrals(Wb, Co, Ca)
    V = O.Integrals(Vb, Co, Ca)
    WV = O.Integrals(WVb, Co, Ca)
    N = Co[0].shape[0]
    F = np.array([[spin_factor(ns, s, sp, s_os, s_ss) for sp in range(ns)] for s in range(ns)])
    lw, lv, lx = W.df_vals, V.df_vals, WV.df_vals
    Sinv = np.block([[abs_p.s_inv_ao_ao, abs_p.s_inv_ao_ri], [abs_p.s_inv_ri_ao, abs_p.s_inv_ri_ri]])
    R = abs_p.s_inv_ri_ri.shape[0]
    Rp = N + R

    def stacked(X, s):
        """Wst: per active orbital j, AO rows (B1 orbital c+j) then RI rows (Bri orbital j)."""
        B1 = X.get_X3idx_one_trans()[s]
        Bri = X.get_X3idx_one_trans_ri()[s]
        o = Co[s].shape[1]
        a = Ca[s].shape[1]
        c = o - a
        M = B1.shape[1]
        out = np.zeros((Rp * a, M))
        for j in range(a):
            out[Rp * j:Rp * j + N] = B1[N * (c + j):N * (c + j + 1)]
            out[Rp * j + N:Rp * (j + 1)] = Bri[R * j:R * (j + 1)]
        return out

    t = O.calculate_tab(W, V)
    tt = O.calculate_ttilde(W, V, t)
    Wst = [stacked(W, s) for s in range(ns)]
    Vst = [stacked(V, s) for s in range(ns)]
    Sop = [np.kron(np.eye(Ca[s].shape[1]), Sinv) for s in range(ns)]
    X = [Wst[s].T @ Sop[s] @ Vst[s] for s in range(ns)]
    XD = WV.get_X_D()

    # ---- adjoints of the M x M intermediates
    tbar, Xbar = [], []
    for s in range(ns):
        tb = sum(0.5 * F[s, sp] * tt[sp] for sp in range(ns))
        ttb = sum(F[sp, s] * (0.5 * t[sp] - X[sp]) for sp in range(ns))
        tbar.append(tb + lw[:, None] * ttb * lv[None, :])
        Xbar.append(-sum(F[s, sp] * tt[sp] for sp in range(ns)))

    def three_index_grads(Xi, which):
        """dE/dJ3_0 and dE/dJ3_ri_0 of W (which=0) or V (which=1) at fixed P2."""
        P2 = Xi.P2
        M = P2.shape[0]
        g3 = np.zeros((N * (N + 1) // 2, M))
        g3ri = np.zeros((R * N, M))
        for s in range(ns):
            o, a = Co[s].shape[1], Ca[s].shape[1]
            c = o - a
            if a == 0:
                continue
            B2o = (V if which == 0 else W).get_X3idx_two_trans()[s]
            B2bar = B2o @ (tbar[s].T if which == 0 else tbar[s])  # (a o) x M
            if which == 0:
                Wstbar = (Sop[s] @ Vst[s]) @ Xbar[s].T
            else:
                Wstbar = (Sop[s] @ Wst[s]) @ Xbar[s]
            B1bar = (Ca[s] @ B2bar.reshape((a, o * M), order="F")).reshape((N * o, M), order="F")
            Brbar = np.zeros((R * a, M))
            for j in range(a):
                B1bar[N * (c + j):N * (c + j + 1)] += Wstbar[Rp * j:Rp * j + N]
                Brbar[R * j:R * (j + 1)] = Wstbar[Rp * j + N:Rp * (j + 1)]
            B10bar = B1bar @ P2.T
            Brbar0 = Brbar @ P2.T
            for A in range(M):
                G = B10bar[:, A].reshape((N, o), order="F") @ Co[s].T
                g3[:, A] += _pack_sym_sum(G)
                g3ri[:, A] += (Brbar0[:, A].reshape((R, a), order="F") @ Ca[s].T).reshape(-1, order="F")
        return g3, g3ri

    gW3, gW3ri = three_index_grads(W, 0)
    gV3, gV3ri = three_index_grads(V, 1)

    # ---- WV: E2 = 1/2 f XD[s] . (L XD[s']), XD = 1/2 ns P2^T J3_0^T lower(D, 2)
    D = O.construct_density(Ca)
    gWV3 = np.zeros_like(WVb.J3_0)
    for s in range(ns):
        XDbar = sum(F[s, sp] * lx * XD[sp] for sp in range(ns))
        vbar = WV.P2 @ XDbar
        gWV3 += 0.5 * ns * np.outer(O.lower(D[s], 2.0), vbar)

    # ---- metrics: dE/dJ2 = -Q [.] Q^T, Q = P2 L
    def sym(A):
        return 0.5 * (A + A.T)

    QW, QV, QX = W.P2 * lw[None, :], V.P2 * lv[None, :], WV.P2 * lx[None, :]
    AW = np.zeros((lw.size, lw.size))
    AV = np.zeros((lv.size, lv.size))
    AX = np.zeros((lx.size, lx.size))
    for s in range(ns):
        for sp in range(ns):
            f = F[s, sp]
            AW += 0.5 * f * (t[sp] * lv[None, :]) @ t[s].T - f * (X[s] * lv[None, :]) @ t[sp].T
            AV += 0.5 * f * (t[s].T * lw[None, :]) @ t[sp] - f * (t[sp].T * lw[None, :]) @ X[s]
            AX += 0.5 * f * np.outer(XD[s], XD[sp])
    gW2 = -sym(QW @ AW @ QW.T)
    gV2 = -sym(QV @ AV @ QV.T)
    gX2 = -sym(QX @ AX @ QX.T)
    return {"W3": gW3, "W3_ri": gW3ri, "W2": gW2, "V3": gV3, "V3_ri": gV3ri, "V2": gV2,
            "WV3": gWV3, "WV2": gX2}


def chunked_three_index_adjoint(Wb, Vb, abs_p, orbitals, occ, n_active, s_os, s_ss, chunk):
    """dE/dJ3_0 and dE/dJ3_ri_0 of W and V (as ``direct_adjoint``) with every
    stacked intermediate formed for at most ``chunk`` orbitals at a time:
    X and t accumulated over orbital chunks (schedule_model.chunked_xab_t); the
    reverse sweep splits by linearity into a B2-bar path over chunks of
    occupied orbitals k (B1bar_k = Ca (B2_other,k tbar^T)) and a Wst-bar path
    over chunks of active orbitals j ((S^-1 Wst_other,j) Xbar^T, whose AO rows
    add to B1bar of orbital c + j and whose RI rows are Bri-bar of j); both
    reach dE/dJ3 through P2^T and the per-aux-function contractions with Co
    (packed symmetric sum) and Ca."""
    from tests import schedule_model as K
    ns = len(orbitals)
    Co = O.occupation_weighted_orbitals(orbitals, occ)
    Ca = O.freeze_core(Co, n_active)
    W = O.Integrals(Wb, Co, Ca)
    V = O.Integrals(Vb, Co, Ca)
    N, M, R = Wb.n_ao, Wb.n_df, Wb.n_ri
    Rp = N + R
    F = np.array([[spin_factor(ns, s, sp, s_os, s_ss) for sp in range(ns)] for s in range(ns)])
    lw, lv = W.df_vals, V.df_vals
    Sinv = np.block([[abs_p.s_inv_ao_ao, abs_p.s_inv_ao_ri], [abs_p.s_inv_ri_ao, abs_p.s_inv_ri_ri]])
    X, t = [], []
    for s in range(ns):
        xs, ts = K.chunked_xab_t(Wb, Vb, Sinv, Co[s], Ca[s], chunk)
        X.append(xs)
        t.append(ts)
    tt = [lw[:, None] * t[s] * lv[None, :] for s in range(ns)]
    tbar, Xbar = [], []
    for s in range(ns):
        tb = sum(0.5 * F[s, sp] * tt[sp] for sp in range(ns))
        ttb = sum(F[sp, s] * (0.5 * t[sp] - X[sp]) for sp in range(ns))
        tbar.append(tb + lw[:, None] * ttb * lv[None, :])
        Xbar.append(-sum(F[s, sp] * tt[sp] for sp in range(ns)))
    out = {}
    for which, (Xi, Yi) in enumerate(((Wb, Vb), (Vb, Wb))):
        P2 = Xi.P2
        g3 = np.zeros((N * (N + 1) // 2, M))
        g3ri = np.zeros((R * N, M))
        for s in range(ns):
            o, a = Co[s].shape[1], Ca[s].shape[1]
            c = o - a
            if a == 0:
                continue
            tb = tbar[s].T if which == 0 else tbar[s]
            xb = Xbar[s].T if which == 0 else Xbar[s]
            # B2-bar path, chunks of occupied orbitals k
            for k0 in range(0, o, chunk):
                k1 = min(o, k0 + chunk)
                nk = k1 - k0
                b2o = K.T3(K.T1(Yi.J3_0, Co[s][:, k0:k1], Yi.P2), Ca[s])  # a nk x M
                b2b = b2o @ tb
                b1b = (Ca[s] @ b2b.reshape((a, nk * M), order="F")).reshape((N * nk, M),
                                                                           order="F")
                b10 = b1b @ P2.T
                for A in range(M):
                    G = b10[:, A].reshape((N, nk), order="F") @ Co[s][:, k0:k1].T
                    g3[:, A] += _pack_sym_sum(G)
            # Wst-bar path, chunks of active orbitals j
            for j0 in range(0, a, chunk):
                j1 = min(a, j0 + chunk)
                nj = j1 - j0
                sy = K._stacked(Yi, Co[s], Ca[s], j0, j1, R)
                ssy = (Sinv @ sy.reshape(Rp, nj * M, order="F")).reshape(Rp * nj, M, order="F")
                wsb = (ssy @ xb).reshape((Rp, nj, M), order="F")
                ao = (wsb[:N].reshape((N * nj, M), order="F")) @ P2.T
                ri = (wsb[N:].reshape((R * nj, M), order="F")) @ P2.T
                for A in range(M):
                    G = ao[:, A].reshape((N, nj), order="F") @ Co[s][:, c + j0:c + j1].T
                    g3[:, A] += _pack_sym_sum(G)
                    g3ri[:, A] += (ri[:, A].reshape((R, nj), order="F") @
                                   Ca[s][:, j0:j1].T).reshape(-1, order="F")
        out["W3" if which == 0 else "V3"] = g3
        out["W3_ri" if which == 0 else "V3_ri"] = g3ri
    return out


def full_energy(W, V, WV, abs_p, orbitals, occ, n_active, s_os, s_ss):
    """Energy with the same-spin (indirect) terms, as uw12_energy with s_ss != 0."""
    return O.form_fock(W, V, WV, abs_p, orbitals, occ, n_active, True, False, s_os,
                       s_ss).energy


def perm_3el(Z, Rp, a, o):
    """P3(Z)[p + Rp i, j + a k] = Z[p + Rp j, i + a k] for Z of shape (Rp a) x (a o)."""
    T = Z.reshape((Rp, a, a, o), order="F")         # (p, row-orbital, col-orbital, k)
    return np.transpose(T, (0, 2, 1, 3)).reshape((Rp * a, a * o), order="F")


def perm_4el(Vm, a, o):
    """P4(V)[i + a l, j + a k] = V[i + a k, j + a l] for V of shape (a o) x (a o)."""
    T = Vm.reshape((a, o, a, o), order="F")          # (i, k_row, j, l_col)
    return np.transpose(T, (0, 3, 2, 1)).reshape((a * o, a * o), order="F")


def indirect_adjoint(Wb, Vb, WVb, abs_p, orbitals, occ, n_active):
    """Gradients of the same-spin energy E_ss with respect to every stored
    integral; uw12_energy's energy is E_direct(s_os, s_ss) + s_ss E_ss, so the
    full gradient is direct_adjoint(...) + s_ss * indirect_adjoint(...).

    With esf = 2 (closed shell) or 1, per spin, all in the metric eigenbasis:
      E2- = -1/2 esf <B2_WV L_WV, B2_WV>              (two_electron.cpp:87-132;
            B2_WV of the active orbitals only)
      E4- = -1/2 esf <W4, P4(V4)>, W4 = B2_W L_W B2_W^T, V4 likewise
                                                      (four_electron.cpp:143-179)
      E3- = esf <YW, P3(ZV)>, YW = Wst_W L_W B2_W^T, ZV = SV_V L_V B2_V^T
            (SV = (I (x) S^-1) Wst)                   (indirect_utils.cpp:101-133)
    Reverse sweep: G_Y = esf P3(ZV), G_Z = esf P3(YW); Wst_W-bar = G_Y B2_W L_W,
    B2_W-bar = G_Y^T Wst_W L_W, SV_V-bar = G_Z B2_V L_V -> Wst_V-bar = (I (x) S^-1)
    SV_V-bar, B2_V-bar = G_Z^T SV_V L_V; G_W4 = -1/2 esf P4(V4): B2_W-bar +=
    2 G_W4 B2_W L_W (and W <-> V); B2_WV-bar = -esf B2_WV L_WV; the transforms
    are then reversed as in direct_adjoint.  Metric: each L between eigenbasis
    factors contributes A += (left factor)^T G (right factor) to
    dE/dJ2 = -sym(Q A Q^T), Q = P2 L."""
    ns = len(orbitals)
    esf = 2.0 if ns == 1 else 1.0
    Co = O.occupation_weighted_orbitals(orbitals, occ)
    Ca = O.freeze_core(Co, n_active)
    W = O.Integrals(Wb, Co, Ca)
    V = O.Integrals(Vb, Co, Ca)
    WVa = O.Integrals(WVb, Ca, Ca)
    N = Co[0].shape[0]
    R = abs_p.s_inv_ri_ri.shape[0]
    Rp = N + R
    Sinv = np.block([[abs_p.s_inv_ao_ao, abs_p.s_inv_ao_ri], [abs_p.s_inv_ri_ao, abs_p.s_inv_ri_ri]])
    lw, lv, lx = W.df_vals, V.df_vals, WVa.df_vals

    def stacked(X, s):
        B1 = X.get_X3idx_one_trans()[s]
        Bri = X.get_X3idx_one_trans_ri()[s]
        o, a = Co[s].shape[1], Ca[s].shape[1]
        c = o - a
        out = np.zeros((Rp * a, B1.shape[1]))
        for j in range(a):
            out[Rp * j:Rp * j + N] = B1[N * (c + j):N * (c + j + 1)]
            out[Rp * j + N:Rp * (j + 1)] = Bri[R * j:R * (j + 1)]
        return out

    def unstack(Wsb, s, M):
        """Wst-bar rows back to (B1-bar rows of the active orbitals, Bri-bar)."""
        o, a = Co[s].shape[1], Ca[s].shape[1]
        c = o - a
        b1 = np.zeros((N * o, M))
        br = np.zeros((R * a, M))
        for j in range(a):
            b1[N * (c + j):N * (c + j + 1)] = Wsb[Rp * j:Rp * j + N]
            br[R * j:R * (j + 1)] = Wsb[Rp * j + N:Rp * (j + 1)]
        return b1, br

    def reverse(Xi, b1bar, brbar, C_occ, C_act, g3, g3ri):
        """B1-bar (N o x M, orbitals C_occ) and Bri-bar (R a x M) to dE/dJ3_0, dE/dJ3_ri_0."""
        P2 = Xi.P2
        M = P2.shape[0]
        o = C_occ.shape[1]
        b10 = b1bar @ P2.T
        for A in range(M):
            G = b10[:, A].reshape((N, o), order="F") @ C_occ.T
            g3[:, A] += _pack_sym_sum(G)
        if brbar is not None and g3ri is not None:
            br0 = brbar @ P2.T
            a = C_act.shape[1]
            for A in range(M):
                g3ri[:, A] += (br0[:, A].reshape((R, a), order="F") @ C_act.T).reshape(-1, order="F")

    MW, MV, MX = lw.size, lv.size, lx.size
    out = {"W3": np.zeros((N * (N + 1) // 2, MW)), "W3_ri": np.zeros((R * N, MW)),
           "V3": np.zeros((N * (N + 1) // 2, MV)), "V3_ri": np.zeros((R * N, MV)),
           "WV3": np.zeros((N * (N + 1) // 2, MX))}
    AW = np.zeros((MW, MW))
    AV = np.zeros((MV, MV))
    AX = np.zeros((MX, MX))
    for s in range(ns):
        o, a = Co[s].shape[1], Ca[s].shape[1]
        if a == 0 or o == 0:
            continue
        B2W = W.get_X3idx_two_trans()[s]
        B2V = V.get_X3idx_two_trans()[s]
        WstW = stacked(W, s)
        SVV = np.kron(np.eye(a), Sinv) @ stacked(V, s)
        # three-electron
        YW = (WstW * lw[None, :]) @ B2W.T
        ZV = (SVV * lv[None, :]) @ B2V.T
        GY = esf * perm_3el(ZV, Rp, a, o)
        GZ = esf * perm_3el(YW, Rp, a, o)
        TY = GY @ B2W
        TZ = GZ @ B2V
        WsbW = TY * lw[None, :]
        WsbV = np.kron(np.eye(a), Sinv) @ (TZ * lv[None, :])
        B2bW = GY.T @ (WstW * lw[None, :])
        B2bV = GZ.T @ (SVV * lv[None, :])
        AW += WstW.T @ TY
        AV += SVV.T @ TZ
        # four-electron
        W4 = (B2W * lw[None, :]) @ B2W.T
        V4 = (B2V * lv[None, :]) @ B2V.T
        GW4 = -0.5 * esf * perm_4el(V4, a, o)
        GV4 = -0.5 * esf * perm_4el(W4, a, o)
        B2bW += 2.0 * (GW4 @ B2W) * lw[None, :]
        B2bV += 2.0 * (GV4 @ B2V) * lv[None, :]
        AW += B2W.T @ GW4 @ B2W
        AV += B2V.T @ GV4 @ B2V
        # back through the transforms of W and V
        for Xi, B2b, Wsb, M, g3, g3ri in ((W, B2bW, WsbW, MW, out["W3"], out["W3_ri"]),
                                          (V, B2bV, WsbV, MV, out["V3"], out["V3_ri"])):
            b1, br = unstack(Wsb, s, M)
            b1 += (Ca[s] @ B2b.reshape((a, o * M), order="F")).reshape((N * o, M), order="F")
            reverse(Xi, b1, br, Co[s], Ca[s], g3, g3ri)
        # two-electron (WV over the active orbitals)
        B2X = WVa.get_X3idx_two_trans()[s]
        B2bX = -esf * B2X * lx[None, :]
        AX += -0.5 * esf * B2X.T @ B2X
        b1 = (Ca[s] @ B2bX.reshape((a, a * MX), order="F")).reshape((N * a, MX), order="F")
        reverse(WVa, b1, None, Ca[s], Ca[s], out["WV3"], None)

    def sym(A):
        return 0.5 * (A + A.T)

    for key, Xi, lam, A in (("W2", W, lw, AW), ("V2", V, lv, AV), ("WV2", WVa, lx, AX)):
        Q = Xi.P2 * lam[None, :]
        out[key] = -sym(Q @ A @ Q.T)
    return out


def blocked_three_index_adjoint(Wb, Vb, abs_p, orbitals, occ, n_active, s_os, s_ss, nb):
    """dE/dJ3_0 and dE/dJ3_ri_0 of W and V (the direct terms, as
    ``direct_adjoint``) computed per block of ``nb`` aux functions of the
    gradient, without any stacked (R' a x M) or B1-sized intermediate:
    for gradient block b of potential X (the other potential Y),
      t path:   B1bar_0[:, b] = Ca (B2_Y (tbar' P2_X^T[:, b]))         (N x o per column)
      Wst path: Z_b = P2_Y (Xbar' P2_X^T[:, b]),  G_b = J3_0^Y Z_b,  H_b = J3_ri_0^Y Z_b,
                Q_b = [sq(G_b) Ca ; H_b Ca] (R' x a per column),  SQ_b = S^-1 Q_b;
      dE/dJ3_0[:, A]    = packed symmetric sum of (B1bar_0[:, A] + SQ_b AO rows at the
                          active orbitals) Co^T,
      dE/dJ3_ri_0[:, A] = SQ_b RI rows Ca^T,
    with tbar' = tbar^T, Xbar' = Xbar^T for X = W and tbar, Xbar for X = V.
    X and t come from orbital chunks (schedule_model.chunked_xab_t)."""
    from tests import schedule_model as K
    ns = len(orbitals)
    Co = O.occupation_weighted_orbitals(orbitals, occ)
    Ca = O.freeze_core(Co, n_active)
    W = O.Integrals(Wb, Co, Ca)
    V = O.Integrals(Vb, Co, Ca)
    N, M, R = Wb.n_ao, Wb.n_df, Wb.n_ri
    Rp = N + R
    F = np.array([[spin_factor(ns, s, sp, s_os, s_ss) for sp in range(ns)] for s in range(ns)])
    lw, lv = W.df_vals, V.df_vals
    Sinv = np.block([[abs_p.s_inv_ao_ao, abs_p.s_inv_ao_ri], [abs_p.s_inv_ri_ao, abs_p.s_inv_ri_ri]])
    X, t = [], []
    for s in range(ns):
        xs, ts = K.chunked_xab_t(Wb, Vb, Sinv, Co[s], Ca[s], max(1, Ca[s].shape[1]))
        X.append(xs)
        t.append(ts)
    tt = [lw[:, None] * t[s] * lv[None, :] for s in range(ns)]
    tbar, Xbar = [], []
    for s in range(ns):
        tb = sum(0.5 * F[s, sp] * tt[sp] for sp in range(ns))
        ttb = sum(F[sp, s] * (0.5 * t[sp] - X[sp]) for sp in range(ns))
        tbar.append(tb + lw[:, None] * ttb * lv[None, :])
        Xbar.append(-sum(F[s, sp] * tt[sp] for sp in range(ns)))
    out = {}
    for which, (Xi, Yi, Xo, Yo) in enumerate(((Wb, Vb, W, V), (Vb, Wb, V, W))):
        P2x, P2y = Xi.P2, Yi.P2
        Mx = P2x.shape[0]
        g3 = np.zeros((N * (N + 1) // 2, Mx))
        g3ri = np.zeros((R * N, Mx))
        for s in range(ns):
            o, a = Co[s].shape[1], Ca[s].shape[1]
            c = o - a
            if a == 0:
                continue
            tb = tbar[s].T if which == 0 else tbar[s]     # M_Y x M_X
            xb = Xbar[s].T if which == 0 else Xbar[s]
            B2y = Yo.get_X3idx_two_trans()[s]              # a o x M_Y
            for b0 in range(0, Mx, nb):
                b1 = min(Mx, b0 + nb)
                cols = b1 - b0
                Pt = P2x.T[:, b0:b1]                       # M_X x cols: P2_X^T[:, b]
                Dt = B2y @ (tb @ Pt)                       # a o x cols
                Zb = P2y @ (xb @ Pt)                       # M_Y x cols
                Gb = Yi.J3_0 @ Zb                          # Np x cols
                Hb = Yi.J3_ri_0 @ Zb                       # R N x cols
                for q in range(cols):
                    b1t = Ca[s] @ Dt[:, q].reshape((a, o), order="F")        # N x o
                    Qao = O.square(Gb[:, q]) @ Ca[s]                          # N x a
                    Qri = Hb[:, q].reshape((R, N), order="F") @ Ca[s]         # R x a
                    SQ = Sinv @ np.vstack([Qao, Qri])                          # R' x a
                    b1t[:, c:] += SQ[:N]
                    g3[:, b0 + q] += _pack_sym_sum(b1t @ Co[s].T)
                    g3ri[:, b0 + q] += (SQ[N:] @ Ca[s].T).reshape(-1, order="F")
        out["W3" if which == 0 else "V3"] = g3
        out["W3_ri" if which == 0 else "V3_ri"] = g3ri
    return out
