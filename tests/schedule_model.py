"""numpy model of the CUDA schedule (test infrastructure).

The CUDA engine restates libuw12's pair loops (parallel_sum_2d over orbital
pairs, parallel_for / parallel_sum over aux functions) as large contractions:
stacked AO+RI intermediates ``Wst`` (R'a x M), ``SV = (I (x) S^-1) Wst``,
X_AB = Wst_W^T SV_V, the combined direct-Fock operator
Y = (k4/2) Σ f t~ - Lw X Lv with per-orbital weights (core 1, active 2), the
t~ dX term through T2 = P2_W Tc P2_V^T, and the same-spin terms as
reduction-batched GEMMs.  This module states exactly that algorithm in numpy
so that it can be checked against the operation-for-operation oracle on the
CPU (tests/test_schedule_model.py); engine.cu follows it step by step.
"""
import numpy as np
from oracle import uw12_oracle as O

def sq_all(P):
    """P: Np x K packed -> N x N x K"""
    Np, K = P.shape
    n = O.n_from_packed(Np)
    r, c = np.tril_indices(n)
    out = np.zeros((n, n, K))
    out[r, c, :] = P
    out[c, r, :] = P
    return out

def T1(J3_0, C, P2):
    # H1[mu + N k, A] = sum_nu sq(J3_0_A)[mu,nu] C[nu,k]
    N, o = C.shape
    if o == 0: return np.zeros((0, J3_0.shape[1]))
    sq = sq_all(J3_0)  # N x N x M
    H = np.einsum('mnA,nk->mkA', sq, C).reshape(N * o, -1, order='F')
    return H @ P2

def T2(J3ri, C, P2, R):
    N, a = C.shape
    M = J3ri.shape[1]
    if a == 0: return np.zeros((0, M))
    J = J3ri.reshape((R, N, M), order='F')
    H = np.einsum('rmA,mi->riA', J, C).reshape(R * a, M, order='F')
    return H @ P2

def T3(B1, Ca):
    N, a = Ca.shape
    M = B1.shape[1]
    o = B1.shape[0] // N
    if a * o == 0: return np.zeros((a * o, M))
    B = B1.reshape((N, o, M), order='F')
    return np.einsum('mi,mkA->ikA', Ca, B).reshape(a * o, M, order='F')

def form_fock(W, V, WV, Sfull_inv, orbitals, occ, n_active, indirect, calc_fock, s_os, s_ss):
    n_spin = len(orbitals)
    Co = O.occupation_weighted_orbitals(orbitals, occ)
    Ca = O.freeze_core(Co, n_active)
    N = W.n_ao; M = W.n_df; R = W.n_ri; Rp = N + R
    Sinv = Sfull_inv  # (ao, ri) order, R' x R'
    f = lambda s, sp: O.get_energy_spin_factor(n_spin, s, sp, s_os, s_ss)
    half = 0.5 if n_spin == 1 else 1.0
    two = 2 if n_spin == 1 else 1
    F = [np.zeros((N, N)) for _ in range(n_spin)]
    E = {}
    do_ind = indirect and s_ss != 0
    # ---------------- 2-el --------------------------------------------------
    lam = WV.df_vals
    XD = []
    for s in range(n_spin):
        D = two * Ca[s] @ Ca[s].T
        d = O.lower(D, 2.0)
        XD.append(0.5 * n_spin * (WV.P2.T @ (WV.J3_0.T @ d)))
    e = 0.0
    for s in range(n_spin):
        vc = np.zeros(M)
        for sp in range(n_spin):
            ff = f(s, sp)
            if ff == 0: continue
            e += 0.5 * ff * XD[s] @ (lam * XD[sp])
            vc += 0.5 * n_spin * ff * lam * XD[sp]
        if calc_fock:
            F[s] += O.square(WV.J3_0 @ (WV.P2 @ vc))
    E['2d'] = e
    if do_ind:
        e = 0.0
        for s in range(n_spin):
            a = Ca[s].shape[1]
            if a == 0: continue
            B1 = T1(WV.J3_0, Ca[s], WV.P2)
            B2 = T3(B1, Ca[s])
            e += -0.5 * two * np.sum(B2 * B2 * lam[None, :])
            if calc_fock:
                r1 = B1.reshape(N, a * M, order='F')
                r1l = (B1 * lam[None, :]).reshape(N, a * M, order='F')
                F[s] += -s_ss * (r1 @ r1l.T)
        E['2i'] = s_ss * e
    # ---------------- transforms ---------------------------------------------
    lw, lv = W.df_vals, V.df_vals
    B1 = {}; Bri = {}; B2 = {}; Wp = {}; SVp = {}
    for s in range(n_spin):
        o = Co[s].shape[1]; a = Ca[s].shape[1]; c = o - a
        for X, nm in ((W, 'W'), (V, 'V')):
            b1 = T1(X.J3_0, Co[s], X.P2)
            bri = T2(X.J3_ri_0, Ca[s], X.P2, R)
            b2 = T3(b1, Ca[s])
            # stacked R' a x M, row p + R' j: p<N ao (B1 orbital c+j), p>=N ri
            st = np.zeros((Rp * a, M))
            st3 = st.reshape((Rp, a, M), order='F')
            st3[:N] = b1.reshape((N, o, M), order='F')[:, c:, :]
            st3[N:] = bri.reshape((R, a, M), order='F')
            st = st3.reshape((Rp * a, M), order='F')
            B1[nm, s] = b1; Bri[nm, s] = bri; B2[nm, s] = b2; Wp[nm, s] = st
            SVp[nm, s] = (Sinv @ st.reshape(Rp, a * M, order='F')).reshape(Rp * a, M, order='F')
    X = [Wp['W', s].T @ SVp['V', s] for s in range(n_spin)]
    t = [B2['W', s].T @ B2['V', s] for s in range(n_spin)]
    tt = [lw[:, None] * t[s] * lv[None, :] for s in range(n_spin)]
    e3 = 0.0; e4 = 0.0
    for s in range(n_spin):
        for sp in range(n_spin):
            ff = f(s, sp)
            e3 -= ff * np.sum(X[s] * tt[sp])
            if ff == 0: continue
            e4 += 0.5 * ff * np.sum(tt[sp] * t[s])
    E['3d'] = e3; E['4d'] = e4
    Fsym = [np.zeros((N, N)) for _ in range(n_spin)]  # pieces symmetrised at end
    if calc_fock:
        kap4 = 2 * half
        for s in range(n_spin):
            o = Co[s].shape[1]; a = Ca[s].shape[1]; c = o - a
            if o == 0: continue
            T4 = sum((f(s, sp) if f(s, sp) != 0 else 0.0) * tt[sp] for sp in range(n_spin))
            Xc = sum(half * f(s, sp) * X[sp] for sp in range(n_spin))
            Xh = lw[:, None] * Xc * lv[None, :]
            Y = (kap4 if a == 0 else 0.5 * kap4) * T4 - Xh
            Z = B1['W', s] @ Y
            Z3 = Z.reshape((N, o, M), order='F').copy()
            if a > 0: Z3[:, c:, :] *= 2.0
            Fsym[s] += Z3.reshape(N, o * M, order='F') @ B1['V', s].reshape(N, o * M, order='F').T
        # tdx (3-el), per sigma'
        for sp in range(n_spin):
            Tc = sum(half * f(s, sp) * tt[s] for s in range(n_spin))
            T2m = W.P2 @ Tc @ V.P2.T
            sm = V.J3_0 @ T2m.T       # Np x M (a index = W side)
            pm = V.J3_ri_0 @ T2m.T    # RN x M
            H = np.zeros((Rp, N, M))
            H[:N] = sq_all(sm)
            H[N:] = pm.reshape((R, N, M), order='F')
            U = np.einsum('pq,qnA->pnA', Sinv, H)
            G = np.zeros((Rp, N, M))
            G[:N] = sq_all(W.J3_0)
            G[N:] = W.J3_ri_0.reshape((R, N, M), order='F')
            Fsym[sp] += -np.einsum('pmA,pnA->mn', G, U)
    # ---------------- indirect 4-el / 3-el -------------------------------------
    if do_ind:
        e4i = 0.0; e3i = 0.0
        for s in range(n_spin):
            o = Co[s].shape[1]; a = Ca[s].shape[1]; c = o - a
            if a == 0 or o == 0: continue
            b2wl = B2['W', s] * lw[None, :]; b2vl = B2['V', s] * lv[None, :]
            W4 = b2wl @ B2['W', s].T; V4 = b2vl @ B2['V', s].T
            W4r = W4.reshape((a, o, a, o), order='F')  # [i,l,j,k]
            V4r = V4.reshape((a, o, a, o), order='F')  # [i,k,j,l]
            e4i += -0.5 * two * np.einsum('iljk,ikjl->', W4r, V4r)
            # 3-el indirect energy
            YW = Wp['W', s] @ b2wl.T   # R'a x ao : [(p,i),(j,k)]
            ZV = SVp['V', s] @ b2vl.T  # [(q,j),(i,k)]
            YWr = YW.reshape((Rp, a, a, o), order='F')  # p,i,j,k
            ZVr = ZV.reshape((Rp, a, a, o), order='F')  # p,j,i,k
            e3i += two * np.einsum('pijk,pjik->', YWr, ZVr)
            if calc_fock:
                # 4-el indirect fock
                W43 = (B1['W', s] * lw[None, :]) @ B2['W', s].T  # No x ao
                V43 = (B1['V', s] * lv[None, :]) @ B2['V', s].T
                W43r = W43.reshape((N, o, a, o), order='F')  # mu, orb, j, k
                V43r = V43.reshape((N, o, a, o), order='F')
                Fi = -2 * np.einsum('mijk,njik->mn', W43r[:, c:, :, :], V43r[:, c:, :, :])
                if c > 0:
                    Ff = -2 * np.einsum('mljk,nkjl->mn', W43r, V43r)
                    Fi = 0.5 * (Fi + Ff)
                Fsym[s] += s_ss * Fi
                # 3-el indirect fock
                Fk = np.zeros((N, N))
                for (Xn, Yn, Xi, Yi) in (('W', 'V', W, V), ('V', 'W', V, W)):
                    lx = Xi.df_vals; ly = Yi.df_vals
                    ZY = SVp[Yn, s] @ (B1[Yn, s] * ly[None, :]).T   # R'a x No
                    xh = Xi.P2 @ (lx[:, None] * B2[Xn, s].T)       # M x ao
                    gao = sq_all(Xi.J3_0 @ xh)                      # N x N x ao
                    gri = (Xi.J3_ri_0 @ xh).reshape((R, N, a * o), order='F')
                    G = np.concatenate([gao, gri], axis=0)          # R' x N x (j,k)
                    G = G.reshape((Rp, N, a, o), order='F')
                    ZYr = ZY.reshape((Rp, a, N, o), order='F')     # q,j,beta,k
                    Fk += np.einsum('pajk,pjbk->ab', G, ZYr)
                Wk = Wp['W', s] @ ((B1['W', s] * lw[None, :]).reshape((N, o, M), order='F')[:, c:, :].reshape(N * a, M, order='F')).T
                Wkr = Wk.reshape((Rp, a, N, a), order='F')   # p,i,beta,j
                ZYV = (SVp['V', s] @ (B1['V', s] * lv[None, :]).T).reshape((Rp, a, N, o), order='F')  # p,j,alpha,k
                Fk += np.einsum('pibj,pjai->ba', Wkr, ZYV[:, :, :, c:])
                Fsym[s] += s_ss * Fk
        E['4i'] = s_ss * e4i; E['3i'] = s_ss * e3i
    Ftot = [O.symmetrise(F[s] + Fsym[s]) for s in range(n_spin)]
    return sum(E.values()), Ftot, E


# ---------------------------------------------------------------------------
# Orbital-chunked form of the direct terms: the stacked intermediates (R' a x
# M per spin and potential) are formed for at most `chunk` orbitals at a time,
# so that their memory is bounded independently of the number of active
# orbitals (the layout a device evaluation of N=2000, M=6000, R=8000 with 170
# active orbitals per spin needs: whole, one stacked tensor is 82 GB).
# ---------------------------------------------------------------------------

def _stacked(Xi, Co_s, Ca_s, j0, j1, R):
    """Rows of Wst for active orbitals j0..j1-1: per orbital, AO rows (B1 of
    occupied column c + j) then RI rows (Bri of active column j)."""
    N = Xi.n_ao
    M = Xi.n_df
    o, a = Co_s.shape[1], Ca_s.shape[1]
    c = o - a
    nj = j1 - j0
    b1 = T1(Xi.J3_0, Co_s[:, c + j0:c + j1], Xi.P2)
    bri = T2(Xi.J3_ri_0, Ca_s[:, j0:j1], Xi.P2, R)
    st3 = np.zeros((N + R, nj, M))
    st3[:N] = b1.reshape((N, nj, M), order='F')
    st3[N:] = bri.reshape((R, nj, M), order='F')
    return st3.reshape(((N + R) * nj, M), order='F')


def chunked_xab_t(W, V, Sinv, Co_s, Ca_s, chunk):
    """X_AB = Wst_W^T (I (x) S^-1) Wst_V accumulated over chunks of active
    orbitals, and t = B2_W^T B2_V accumulated over chunks of occupied orbitals
    (B2 rows i + a k: the k-chunk's rows are formed from its B1 columns)."""
    N, R, M = W.n_ao, W.n_ri, W.n_df
    Rp = N + R
    o, a = Co_s.shape[1], Ca_s.shape[1]
    X = np.zeros((M, M))
    t = np.zeros((M, M))
    for j0 in range(0, a, chunk):
        j1 = min(a, j0 + chunk)
        nj = j1 - j0
        sw = _stacked(W, Co_s, Ca_s, j0, j1, R)
        sv = _stacked(V, Co_s, Ca_s, j0, j1, R)
        svs = (Sinv @ sv.reshape(Rp, nj * M, order='F')).reshape(Rp * nj, M, order='F')
        X += sw.T @ svs
    for k0 in range(0, o, chunk):
        k1 = min(o, k0 + chunk)
        b2w = T3(T1(W.J3_0, Co_s[:, k0:k1], W.P2), Ca_s)
        b2v = T3(T1(V.J3_0, Co_s[:, k0:k1], V.P2), Ca_s)
        t += b2w.T @ b2v
    return X, t


def chunked_direct_fock(W, V, Co_s, a, Y, chunk):
    """Σ_k (B1_W Y)_k (B1_V)_k^T (active orbitals k >= c weighted 2), with B1 of
    W and V formed for at most `chunk` occupied orbitals at a time."""
    N = W.n_ao
    o = Co_s.shape[1]
    c = o - a
    F = np.zeros((N, N))
    for k0 in range(0, o, chunk):
        k1 = min(o, k0 + chunk)
        nk = k1 - k0
        b1w = T1(W.J3_0, Co_s[:, k0:k1], W.P2)
        b1v = T1(V.J3_0, Co_s[:, k0:k1], V.P2)
        Z3 = (b1w @ Y).reshape((N, nk, -1), order='F').copy()
        for idx in range(nk):
            if a > 0 and k0 + idx >= c:
                Z3[:, idx, :] *= 2.0
        F += Z3.reshape(N, -1, order='F') @ b1v.reshape(N, -1, order='F').T
    return F
