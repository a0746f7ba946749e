"""CPU oracle of the iTEBD gates path (test infrastructure: only tests/ use
it, as the checker of the device implementation).

Restates the reference's infinite-chain imaginary-time evolution in Vidal
form with a two-site unit cell (TensorNetworksImp/iTEBD):
- gates exp(-dt h) of the two-site Hamiltonian (Hamiltonian::GetExponentH,
  TensorNetworks/Hamiltonian.C:22-44), second-order Trotter sequence
  dt/2, dt, dt/2 (iTEBDGates::InitGates, iTEBDGates.C:21-54);
- each gate on the bond between the current sites A and B
  (iTEBDStateImp::Apply(MultigateType), iTEBDStateImp_iTime.C:119-135):
  theta = lB GA[ma] lA GB[mb] lB (ContractTheta lAlBl,
  iTEBDStateImp_Contractions.C:24-84), theta'[na,nb] = sum expH theta[ma,mb],
  reshaped with row i + D*na and column j + D*nb (ReshapeForSVD,
  iTEBDStateImp_OrthoNorm.C:24-42), SVD, compression (eps = 1e-7 for all but
  the last two gates, Dmax after them; SVCompressorImp.C:19-73), new lambdaA
  normalised (Bond::SetSingularValues) and GA = lB^-1 U, GB = Vt lB^-1
  (Unpack, iTEBDStateImp_OrthoNorm.C:205-270); the next gate acts on the
  other bond (ReCenter).
- energy per bond: <theta|h|theta>/<theta|theta> with theta = lB GA lA GB lB,
  averaged over the two bonds.  (The reference re-orthogonalises the state
  and evaluates the iMPO expectation; for a converged near-canonical state the
  two agree to the truncation level.)"""
import numpy as np

from . import oracle as O


def gate(S, Jxy, Jz, hz, dt):
    """exp(-dt h12) as (d^2, d^2) with rows (ma*d + mb), columns (na*d + nb)."""
    h = O.local_h12(S, Jxy, Jz, hz)
    w, U = np.linalg.eigh(0.5 * (h + h.T))
    return (U * np.exp(-dt * w)) @ U.T


def compress(s, Dmax, eps):
    """SVCompressorImp::Compress: kept count and the rescaled kept values."""
    s = np.asarray(s, dtype=np.float64)
    n = s.size
    if eps > 0:
        tail = np.cumsum((s * s)[::-1])[::-1]  # tail[k] = sum_{i>=k} s_i^2
        keep = n
        for k in range(1, n + 1):
            if k == n or tail[k] < eps:
                keep = k
                break
        if Dmax > 0:
            keep = min(keep, Dmax)
    else:
        keep = min(n, Dmax) if Dmax > 0 else n
    s2b = float(np.sum(s * s))
    s2a = float(np.sum(s[:keep] ** 2))
    sk = s[:keep] * (s2b / s2a if s2a > 0 else 1.0)
    return keep, sk


def apply_gate(GA, GB, lA, lB, G, Dmax, eps):
    d = GA.shape[0]
    Dl = lB.size
    X = lB[None, :, None] * GA * lA[None, None, :]      # (d, Dl, Dm)
    Y = GB * lB[None, None, :]                          # (d, Dm, Dl)
    th0 = np.einsum("aij,bjk->abik", X, Y)              # (ma, mb, Dl, Dl)
    th = np.einsum("pq,qik->pik", G.T, th0.reshape(d * d, Dl, Dl)).reshape(d, d, Dl, Dl)  # (na, nb, i, k)
    M = np.empty((d * Dl, d * Dl))
    for na in range(d):
        for nb in range(d):
            M[na * Dl:(na + 1) * Dl, nb * Dl:(nb + 1) * Dl] = th[na, nb]
    U, s, Vt = np.linalg.svd(M, full_matrices=False)
    keep, sk = compress(s, Dmax, eps)
    lA_new = sk / np.linalg.norm(sk)
    GA_new = np.empty((d, Dl, keep))
    GB_new = np.empty((d, keep, Dl))
    for n in range(d):
        GA_new[n] = U[n * Dl:(n + 1) * Dl, :keep] / lB[:, None]
        GB_new[n] = Vt[:keep, n * Dl:(n + 1) * Dl] / lB[None, :]
    return GA_new, GB_new, lA_new


def bond_energy(GA, GB, lA, lB, h):
    d = GA.shape[0]
    X = lB[None, :, None] * GA * lA[None, None, :]
    Y = GB * lB[None, None, :]
    th = np.einsum("aij,bjk->abik", X, Y).reshape(d * d, -1)
    return float(np.einsum("pk,pq,qk->", th, h, th) / np.einsum("pk,pk->", th, th))


class State:
    """Two-site unit cell: G[0] on site 1, G[1] on site 2; l[0] = bond 1-2, l[1] = bond 2-1."""

    def __init__(self, S, D, seed=1):
        self.S = S
        self.d = int(round(2 * S + 1))
        rng = np.random.default_rng(seed)
        self.G = [rng.uniform(-1, 1, size=(self.d, D, D)) for _ in range(2)]
        self.l = [np.ones(D) / np.sqrt(D), np.ones(D) / np.sqrt(D)]

    def gate_on(self, b, G, Dmax, eps):
        """Gate on bond b (0: sites 1-2, 1: sites 2-1)."""
        A, B = (0, 1) if b == 0 else (1, 0)
        GA, GB, lnew = apply_gate(self.G[A], self.G[B], self.l[b], self.l[1 - b], G, Dmax, eps)
        self.G[A], self.G[B], self.l[b] = GA, GB, lnew

    def step(self, gates, Dmax):
        """One Trotter step: gate i on bond i mod 2; eps-only compression for
        all but the last two gates (1e-7), then Dmax (eps 1e-16)."""
        n = len(gates)
        for i, G in enumerate(gates):
            if i + 1 <= n - 2:
                self.gate_on(i % 2, G, 0, 1e-7)
            else:
                self.gate_on(i % 2, G, Dmax, 1e-16)

    def energy(self, h):
        e0 = bond_energy(self.G[0], self.G[1], self.l[0], self.l[1], h)
        e1 = bond_energy(self.G[1], self.G[0], self.l[1], self.l[0], h)
        return 0.5 * (e0 + e1)


def find_ground_state(S, D, dts, max_iter, Jxy=1.0, Jz=1.0, hz=0.0, seed=1, eps_factor=5e-5):
    """Second-order iTEBD over the dt schedule; each line runs until the bond
    values change by at most eps_factor*dt or max_iter steps."""
    st = State(S, D, seed)
    h = O.local_h12(S, Jxy, Jz, hz)
    steps = []
    for dt in dts:
        gates = [gate(S, Jxy, Jz, hz, dt / 2), gate(S, Jxy, Jz, hz, dt), gate(S, Jxy, Jz, hz, dt / 2)]
        n = 0
        for n in range(1, max_iter + 1):
            old = [x.copy() for x in st.l]
            st.step(gates, D)
            dl = max(np.abs(o - x).max() if o.size == x.size else 1.0 for o, x in zip(old, st.l))
            if dl <= eps_factor * dt:
                break
        steps.append(n)
    return st.energy(h), st, steps


def expectation(st, h):
    """Energy per bond from the unit-cell transfer-matrix fixed points (the
    infinite-chain expectation value, without assuming canonical form)."""
    from scipy.sparse.linalg import LinearOperator, eigs
    d = st.d
    A1 = st.G[0] * st.l[0][None, None, :]   # site 1 then bond 1-2
    A2 = st.G[1] * st.l[1][None, None, :]   # site 2 then bond 2-1
    D = A2.shape[2]

    def cell(P, Q):  # two-site blocks P[m1] Q[m2]
        return np.einsum("aij,bjk->abik", P, Q)

    def fixed_points(P, Q):
        B = cell(P, Q).reshape(d * d, D, D)
        Lop = LinearOperator((D * D, D * D), matvec=lambda v: np.einsum(
            "pij,ik,pkl->jl", B, v.reshape(D, D), B).ravel())
        Rop = LinearOperator((D * D, D * D), matvec=lambda v: np.einsum(
            "pij,jl,pkl->ik", B, v.reshape(D, D), B).ravel())
        wl, vl = eigs(Lop, k=1, which="LM", tol=1e-14)
        wr, vr = eigs(Rop, k=1, which="LM", tol=1e-14)
        return np.real(vl[:, 0]).reshape(D, D), np.real(vr[:, 0]).reshape(D, D), B

    es = []
    for P, Q in ((A1, A2), (A2, A1)):
        lft, rgt, B = fixed_points(P, Q)
        num = np.einsum("ik,pq,pij,qkl,jl->", lft, h, B, B, rgt)
        den = np.einsum("ik,pij,pkl,jl->", lft, B, B, rgt)
        es.append(num / den)
    return float(0.5 * (es[0] + es[1]))


# ---------------------------------------------------------------------------
# Re-orthogonalisation between schedule lines and the reference's line driver
# ---------------------------------------------------------------------------
def norm_matrices(gam, lam):
    """GetNormMatrix (iTEBDStateImp_Contractions.C:293-333) of gamma*lambda
    (DRight: sum_n M_n M_n^T) and of lambda*gamma (DLeft: sum_n M_n^T M_n)."""
    Mr = gam * lam[None, None, :]
    Ml = lam[None, :, None] * gam
    Vr = np.einsum("nij,nkj->ik", Mr, Mr)
    Vl = np.einsum("nij,nik->jk", Ml, Ml)
    return Vr, Vl


def factor(V):
    """Factor (iTEBDStateImp_OrthoNorm.C:486-509): V = X X^T with X = U sqrt(e),
    Xinv = sqrt(e)^-1 U^T, from the eigen-decomposition of the symmetrised V."""
    e, U = np.linalg.eigh(0.5 * (V + V.T))
    X = U * np.sqrt(e)[None, :]
    Xinv = (U / np.sqrt(e)[None, :]).T
    return X, Xinv


def orthogonalize_gamma(gam, lam, eps, max_iter):
    """OrthogonalizeI(gamma, lambda, eps, maxIter), iTEBDStateImp_OrthoNorm.C:511-637:
    the iterative re-orthogonalisation of Phien, McCulloch and Vidal (PRB 91,
    115137, 2015).  gam is (d*d, D, D), lam (D,).  Returns (gam, lam, bailed)."""
    gam = gam.copy()
    lam = lam.copy()
    er = 1.0
    for it in range(max_iter):
        Vr, Vl = norm_matrices(gam, lam)
        if min(np.abs(np.diag(Vr)).min(), np.abs(np.diag(Vl)).min()) < 1e-10:
            return gam, lam, True       # singular: bail out without the final normalisation (:547-554)
        er, el = Vr[0, 0], Vl[0, 0]
        Vr = Vr / er
        Vl = Vl / el
        gam = gam / np.sqrt(el)
        X, Xinv = factor(Vr)
        Yd, Ydinv = factor(Vl)
        if np.isnan(X).any() or np.isnan(Yd).any():
            return gam, lam, True
        YT, YTinv = Yd.T, Ydinv.T
        U, lp, VT = np.linalg.svd(YT @ (lam[:, None] * X))
        lp = lp / np.sqrt(np.dot(lp, lp))
        VX, YU = VT @ Xinv, YTinv @ U
        gam = np.einsum("ij,njk,kl->nil", VX, gam, YU)
        deltal = np.abs(lam - lp).max()
        lam = lp
        if deltal < eps:
            break
    gam = gam / np.sqrt(er)
    return gam, lam, False


def unpack_orthonormal(st, gam, Dmax, eps_compress=1e-16):
    """UnpackOrthonormal (iTEBDStateImp_OrthoNorm.C:148-200) at centre 1:
    lambdaB gamma[na + d nb] lambdaB reshaped (row i + D na, column j + D nb),
    SVD, SVCompressor(Dmax, eps), lambdaA = s/|s|, GA = lB^-1 P, GB = Q lB^-1."""
    d = st.d
    lB = st.l[1]
    D = lB.size
    M = np.empty((d * D, d * D))
    for nb in range(d):
        for na in range(d):
            M[na * D:(na + 1) * D, nb * D:(nb + 1) * D] = lB[:, None] * gam[na + d * nb] * lB[None, :]
    U, s, Vt = np.linalg.svd(M, full_matrices=False)
    keep, sk = compress(s, Dmax, eps_compress)
    st.l[0] = sk / np.linalg.norm(sk)
    st.G[0] = np.stack([U[n * D:(n + 1) * D, :keep] / lB[:, None] for n in range(d)])
    st.G[1] = np.stack([Vt[:keep, n * D:(n + 1) * D] / lB[None, :] for n in range(d)])


def orthogonalize_i(st, Dmax, eps, max_iter=100):
    """iTEBDStateImp::OrthogonalizeI(comp, eps, niter) (iTEBDStateImp_OrthoNorm.C:110-128)
    at centre 1: gamma[na + d nb] = GA[na] lA GB[nb] (ContractAlB), the
    iteration above on (gamma, lambdaB), lambdaB := the result normalised,
    then UnpackOrthonormal with the (Dmax, 1e-16) compressor."""
    d = st.d
    GA, GB, lA = st.G[0], st.G[1], st.l[0]
    gam = np.stack([(GA[na] * lA[None, :]) @ GB[nb] for nb in range(d) for na in range(d)])
    # the stack above runs nb outer, na inner: index na + d*nb, as ContractAlB
    gam, lam, _ = orthogonalize_gamma(gam, st.l[1], eps, max_iter)
    st.l[1] = lam / np.linalg.norm(lam)
    unpack_orthonormal(st, gam, Dmax)


def grow(st, D):
    """IncreaseBondDimensions (iTEBDStateImp.C:63, MPSSite::NewBondDimensions,
    Bond::NewBondDimension Bond.C:60-84): Gammas zero-padded to D x D, bond
    values padded with min(s)/10 and renormalised."""
    for b in range(2):
        l = st.l[b]
        if l.size < D:
            st.l[b] = np.concatenate([l, np.full(D - l.size, l.min() / 10.0)])
            st.l[b] /= np.linalg.norm(st.l[b])
    for s in range(2):
        g = st.G[s]
        out = np.zeros((st.d, D, D))
        out[:, :g.shape[1], :g.shape[2]] = g
        st.G[s] = out


def find_ground_state_lines(S, Dstart, Dmax, deltaD, dts, max_iter, Jxy=1.0, Jz=1.0, hz=0.0, seed=1,
                            eps_factor=5e-5, orth_iter=100):
    """iTEBDStateImp::FindiTimeGroundState(H, iH, H2, line), iTEBDStateImp_iTime.C:44-104,
    over the schedule of iTEBDTests.C (MakeSchedule: dt lines, dlambda epsilon
    eps_factor*dt, D grown from the current D to Dmax by deltaD inside each
    line): per line OrthogonalizeI (eps dt^2/1000, 1e-13 for dt = 0), then
    for each D the second-order steps until both bond vectors change by at
    most eps_factor*dt, then OrthogonalizeI again.  Returns (E, state, steps)."""
    st = State(S, Dstart, seed)
    h = O.local_h12(S, Jxy, Jz, hz)
    steps = []
    for dt in dts:
        gates = [gate(S, Jxy, Jz, hz, dt / 2), gate(S, Jxy, Jz, hz, dt), gate(S, Jxy, Jz, hz, dt / 2)]
        eps_orth = 1e-13 if dt == 0.0 else dt * dt / 1000.0
        Dcur = max(st.l[0].size, st.l[1].size)
        orthogonalize_i(st, Dcur, eps_orth, orth_iter)
        D = Dcur
        while D <= Dmax:
            if D > Dcur:
                grow(st, D)
            n = 0
            for n in range(1, max_iter + 1):
                old = [x.copy() for x in st.l]
                st.step(gates, D)
                dl = max(np.abs(o - x).max() if o.size == x.size else 1.0 for o, x in zip(old, st.l))
                if dl <= eps_factor * dt:
                    break
            steps.append(n)
            orthogonalize_i(st, D, eps_orth, orth_iter)
            Dcur = D
            D += deltaD
    return expectation(st, h), st, steps
