"""Seeded synthetic problems for the parity tests, built with the oracle (CPU).

A problem is a Dyson equation [i d/dt + mu - H(t)] G - Sigma*G = 1 with
  Sigma = lam^2 * G_bath, G_bath = green_from_H of a random Hermitian s x s bath matrix,
  H(t)  = h0 + f(t) h1 for t >= 0 and H(-1) = h0 (h0, h1 random Hermitian),
solved by the oracle with dyson_mat (fixpoint) -> dyson_start -> dyson_timestep.
"""
import numpy as np

from nessi_b200 import herm_matrix, function


def rand_herm(rng, s, scale):
    x = rng.normal(0, scale, (s, s)) + 1j * rng.normal(0, scale, (s, s))
    return (x + x.conj().T) / 2


def make_sigma(O, rng, nt, ntau, s, sig, beta, h, lam=0.5):
    hb = rand_herm(rng, s, 0.7) + np.diag(rng.uniform(-1, 1, s))
    S = herm_matrix(nt, ntau, s, sig)
    O.green_from_H(S, 0.0, hb, beta, h)
    for t in range(-1, nt + 1):
        S.smul(t, lam * lam)
    return S


def make_H(rng, nt, s, h):
    h0 = rand_herm(rng, s, 0.8)
    h1 = rand_herm(rng, s, 0.4)
    H = function(nt, s)
    H.set_value(-1, h0)
    for t in range(nt + 1):
        H.set_value(t, h0 + np.sin(1.3 * t * h) * h1)
    return H


def solve_oracle(O, G, H, Sigma, mu, beta, h, k, nt_stop=None):
    """Full oracle solution; returns G (all steps) and a copy after the bootstrap."""
    O.dyson_mat(G, Sigma, mu, H, beta, k)
    O.dyson_start(G, mu, H, Sigma, beta, h, k)
    G0 = G.copy()
    nt = G.nt if nt_stop is None else nt_stop
    for n in range(k + 1, nt + 1):
        O.dyson_timestep(n, G, mu, H, Sigma, beta, h, k)
    return G, G0


def rel_err(a, b):
    """max|a - b| / max|b| (0 when both vanish)."""
    den = np.max(np.abs(b)) if b.size else 0.0
    num = np.max(np.abs(a - b)) if a.size else 0.0
    return 0.0 if den == 0 else num / den


def component_errors(Gg, Go, n0, n1):
    """Relative errors of ret/les/tv over time steps n0..n1."""
    out = {}
    rr = [Gg.ret_row(n) for n in range(n0, n1 + 1)]
    ro = [Go.ret_row(n) for n in range(n0, n1 + 1)]
    out["ret"] = rel_err(np.concatenate(rr), np.concatenate(ro))
    lr = [Gg.les_col(n) for n in range(n0, n1 + 1)]
    lo = [Go.les_col(n) for n in range(n0, n1 + 1)]
    out["les"] = rel_err(np.concatenate(lr), np.concatenate(lo))
    out["tv"] = rel_err(Gg.tv[n0:n1 + 1], Go.tv[n0:n1 + 1])
    return out


def make_lattice(O, nkx, nky, nt, ntau, beta, h, u_max, t_ramp, u_mat=0.0, mu=0.0):
    """Square-lattice k-points eps_k = -2(cos kx + cos ky) (size1 = 1) with free initial G_k
    (green_from_H) and a linear ramp U(t) = u_max min(t h / t_ramp, 1), U(-1) = u_mat.
    Returns (Gs, Hs, U) with Hs of shape (nk, nt+2, 1, 1) and U of shape (nt+2, 1)."""
    ks = [(2 * np.pi * i / nkx - np.pi, 2 * np.pi * j / nky - np.pi) for i in range(nkx) for j in range(nky)]
    Gs, Hs = [], []
    for kx, ky in ks:
        e = -2.0 * (np.cos(kx) + np.cos(ky))
        G = herm_matrix(nt, ntau, 1, -1)
        O.green_from_H(G, mu, np.array([[e]]), beta, h)
        Gs.append(G)
        Hs.append(np.full((nt + 2, 1, 1), e, np.complex128))
    U = np.zeros((nt + 2, 1), np.complex128)
    U[0, 0] = u_mat
    for t in range(nt + 1):
        U[t + 1, 0] = u_max * min(t * h / t_ramp, 1.0)
    return Gs, np.array(Hs), U


def u_matrices(U):
    """(nt+2, s) diagonal values -> (nt+2, s, s) cntr::function blocks for the oracle."""
    nt2, s = U.shape
    out = np.zeros((nt2, s, s), np.complex128)
    for i in range(s):
        out[:, i, i] = U[:, i]
    return out


# ---- problems of the benchmark configurations at full shape --------------------------------
def fingerprints(G, nt, nproj=4):
    """Projections of every time-step slice of G: for each t the ret row G^R(t, 0..t), the les
    column G^<(0..t, t) and the tv row G^tv(t, .), flattened and projected onto nproj fixed
    complex vectors v_j[i] = exp(2 pi i (i+1) alpha_j) / L of unit 1-norm, so that
    |f - f_ref| <= max|x - x_ref| element by element.  Returns {comp: (nt+1, nproj) complex,
    comp + "_max": max|x| over all slices}."""
    alphas = np.array([0.6180339887498949, 0.4142135623730951, 0.7320508075688772, 0.2360679774997897])[:nproj]
    out = {}
    for comp in ("ret", "les", "tv"):
        f = np.zeros((nt + 1, nproj), np.complex128)
        mx = 0.0
        for t in range(nt + 1):
            x = (G.ret_row(t) if comp == "ret" else G.les_col(t) if comp == "les" else G.tv[t]).reshape(-1)
            L = x.size
            v = np.exp(2j * np.pi * np.outer(alphas, np.arange(1, L + 1))) / L
            f[t] = v @ x
            mx = max(mx, float(np.max(np.abs(x))))
        out[comp] = f
        out[comp + "_max"] = mx
    return out


def fingerprint_errors(fp, ref):
    """max_t |f - f_ref| / max|x_ref| per component (a lower bound of the relative error of the
    slices themselves)."""
    return {c: float(np.max(np.abs(fp[c] - ref[c])) / ref[c + "_max"]) for c in ("ret", "les", "tv")}


def config3_problem(s, nt, seed, ntau=400, beta=10.0, h=0.01, V=0.7, k=5):
    """One problem of the uneven batch (config 3): h = (X + X^H)/2, X complex N(0, 0.5^2), a
    rank-1 quench u u^H (u complex N(0, 0.3^2)) switched on at t = 0, Sigma = V^2 G_bath (x) 1_s;
    bootstrap = the free propagator of h (mat and steps 0..k).  Returns (desc, H, Sigma, boot)."""
    from nessi_b200 import equilibrium as eq
    from nessi_b200.workloads import bootstrap_free
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 0.5, (s, s)) + 1j * rng.normal(0, 0.5, (s, s))
    h0 = (x + x.conj().T) / 2
    u = rng.normal(0, 0.3, s) + 1j * rng.normal(0, 0.3, s)
    H = np.zeros((nt + 2, s, s), np.complex128)
    H[0] = h0
    H[1:] = h0 + np.outer(u, u.conj())
    Sig = eq.kron_identity(eq.semicircle_bath(nt, ntau, beta, h), s, V * V)
    boot = bootstrap_free(h0, 0.0, beta, h, k, ntau)
    desc = dict(nt=nt, ntau=ntau, size1=s, sig=-1, solve_order=k, sigma_group=0, beta=beta, h=h, mu=0.0)
    return desc, H, Sig, boot


def boot_to_full(boot, desc, k=5):
    """herm_matrix(nt) holding mat and steps 0..k of a bootstrap."""
    G = herm_matrix(desc["nt"], desc["ntau"], desc["size1"], desc["sig"])
    G.mat[...] = boot.mat
    for t in range(k + 1):
        G.set_timestep_data(t, boot.get_timestep(t))
    return G
