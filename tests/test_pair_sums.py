"""The algebra the grouped N-band kernel's Fourier sums rest on, checked on
the CPU with the SyntheticWannier tables: pairing every lattice vector R with
-R, sig = h_R + h_-R and tau = i (h_R - h_-R) give

    h_R e^{iKR} + h_-R e^{-iKR} = c sig + s tau,               e^{iKR} = c + i s
    R_a (h_R e^{iKR} - h_-R e^{-iKR}) = R_a (c (-i tau) + s (i sig)),

so one phase per pair reproduces H0(K) = sum_R h_R e^{iKR} and
S_a(K) = sum_R R_a h_R e^{iKR} (R = 0 stands alone with h_-R = 0); and E.D
summed from a table of E_x d_x + E_y d_y equals E_x D_x + E_y D_y."""
import numpy as np

from antelope_b200 import wannier


def model(seed=4):
    g = wannier.generate(seed)
    m = wannier.synthetic_model(g)
    L = np.asarray(m["lattice"]).reshape(2, 2)
    vec = m["R"] @ L   # Cartesian lattice vectors
    return m, vec


def pairs(R):
    """(r, partner or -1) in the order the host builds them: the first
    vector of each pair, its negative found among the later ones."""
    used = np.zeros(len(R), bool)
    out = []
    for r in range(len(R)):
        if used[r]:
            continue
        used[r] = True
        mate = -1
        for r2 in range(r + 1, len(R)):
            if not used[r2] and R[r2, 0] == -R[r, 0] and R[r2, 1] == -R[r, 1]:
                mate = r2
                used[r2] = True
                break
        out.append((r, mate))
    return out


def test_pair_sums_reproduce_the_fourier_series():
    m, vec = model()
    h, d = m["h"], m["d"]
    pr = pairs(m["R"])
    assert len(pr) == len(vec) // 2 + 1   # every vector pairs up but R = 0
    rng = np.random.default_rng(7)
    for K in rng.normal(scale=0.7, size=(6, 2)):
        ph = np.exp(1j * vec @ K)
        H = np.einsum("r,rij->ij", ph, h)
        Sx = np.einsum("r,r,rij->ij", vec[:, 0], ph, h)
        E = rng.normal(size=2) * 0.01
        ED = np.einsum("r,rij->ij", ph, E[0] * d[:, 0] + E[1] * d[:, 1])
        Hp = np.zeros_like(H)
        Sp = np.zeros_like(H)
        EDp = np.zeros_like(H)
        for r, mate in pr:
            c, s = np.cos(vec[r] @ K), np.sin(vec[r] @ K)
            hm = h[mate] if mate >= 0 else 0.0
            sig, tau = h[r] + hm, 1j * (h[r] - hm)
            Hp += c * sig + s * tau
            Sp += vec[r, 0] * (c * (-1j * tau) + s * (1j * sig))
            e_r = E[0] * d[r, 0] + E[1] * d[r, 1]
            e_m = E[0] * d[mate, 0] + E[1] * d[mate, 1] if mate >= 0 else 0.0
            EDp += c * (e_r + e_m) + s * 1j * (e_r - e_m)
        scale = np.abs(H).max()
        assert np.abs(Hp - H).max() < 1e-14 * scale
        assert np.abs(Sp - Sx).max() < 1e-14 * max(scale, np.abs(Sx).max())
        assert np.abs(EDp - ED).max() < 1e-14 * max(np.abs(ED).max(), 1e-300)
        assert np.abs(H - H.conj().T).max() < 1e-14 * scale
