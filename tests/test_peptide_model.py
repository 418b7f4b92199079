"""The peptide model of the host layer (hamiltonian = peptide) against a numpy statement of
the reference's build_peptide_hamiltonian (src/hamiltonian.f90:195-260): the alpha-helix
geometry phi_n = n dphi, r_n = (R cos phi_n, R sin phi_n, (n-1) rise), the on-site dipole
ramp, hoppings t exp(-(l - l1)/decay) up to hop_range, the radial SOC of every bond (its
lambda_j = 2 lambda exp(..) cos((phi_m - phi_i)/2) along rhat x dhat) or the torsion SOC of
(i, i+2), and the Hermitian completion from the upper triangle. Input keys and defaults of
src/input_output.f90:75-80. CPU only: the model is built on the host."""
import numpy as np
import pytest

import quichotte_b200 as qb

COMMON = """T = 300.d0
V = -0.5d0
Vf = 0.5d0
delv = 0.25
mu = 0
order = 2
dw = 1
up = 1
delta = 0.05
E_CC = 0.3d0
t_hop = -0.7d0
U_int = 0.8d0
GammaL_up = 0.5d0
GammaL_down = 0.4d0
GammaR = 0.5d0
"""


def peptide_h(Nat, twist, rise, R, hand, hop_range, decay, t_hop, lamb, E_CC, ramp, soc_model):
    """H (2 Nat x 2 Nat, spin fastest) of the peptide model, written from its equations."""
    No = 2 * Nat
    dphi = hand * twist * np.pi / 180.0
    phi = dphi * np.arange(1, Nat + 1)
    rs = np.stack([R * np.cos(phi), R * np.sin(phi), rise * np.arange(Nat)], axis=1)
    l1 = np.linalg.norm(rs[1] - rs[0])
    H = np.zeros((No, No), np.complex128)

    def soc_block(i, m, lam, v, add):
        # spin block between sites i and m (0-based): i lam (v . sigma)
        blk = 1j * lam * np.array([[v[2], v[0] - 1j * v[1]], [v[0] + 1j * v[1], -v[2]]])
        if add:
            H[2 * i:2 * i + 2, 2 * m:2 * m + 2] += blk
        else:
            H[2 * i:2 * i + 2, 2 * m:2 * m + 2] = blk

    for i in range(Nat):
        H[2 * i, 2 * i] = H[2 * i + 1, 2 * i + 1] = E_CC + ramp * (i / (Nat - 1) - 0.5)
    if soc_model == "torsion":
        for i in range(Nat - 2):
            d1 = rs[i] - rs[i + 1]
            d2 = rs[i] - rs[i + 2]
            v = np.cross(d1 / np.linalg.norm(d1), d2 / np.linalg.norm(d2))
            soc_block(i, i + 2, lamb, v, add=False)
    for j in range(1, min(hop_range, Nat - 1) + 1):
        for i in range(Nat - j):
            m = i + j
            d = rs[m] - rs[i]
            l = np.linalg.norm(d)
            fac = np.exp(-(l - l1) / decay)
            H[2 * i, 2 * m] += t_hop * fac
            H[2 * i + 1, 2 * m + 1] += t_hop * fac
            if soc_model == "radial":
                pb = 0.5 * (phi[i] + phi[m])
                nu = np.cross([np.cos(pb), np.sin(pb), 0.0], d / l)
                soc_block(i, m, 2.0 * lamb * fac * np.cos(0.5 * (phi[m] - phi[i])), nu, add=True)
    U = np.triu(H)
    return U + np.conj(np.triu(U, 1)).T  # the lower triangle from the upper one


@pytest.mark.parametrize("soc_model,hand,hop_range,ramp", [("radial", 1, 1, 0.0), ("radial", -1, 3, 0.2),
                                                            ("torsion", 1, 2, -0.1), ("torsion", -1, 4, 0.05)])
def test_peptide_hamiltonian_matches_its_equations(tmp_path, soc_model, hand, hop_range, ramp):
    Nat, twist, rise, R, decay, lamb = 11, 100.0, 1.5, 2.3, 0.8, 0.02
    keys = (f"hamiltonian = peptide\nN_sites = {Nat}\nhel_radius = {R}\nhand = {hand}\npep_twist = {twist}\n"
            f"pep_rise = {rise}\nhop_range = {hop_range}\nhop_decay = {decay}\nsoc_model = {soc_model}\n"
            f"dipole_ramp = {ramp}\nlamb = {lamb}\n")
    (tmp_path / "input.dat").write_text(COMMON + keys)
    m = qb.Model.load(str(tmp_path))
    ref = peptide_h(Nat, twist, rise, R, hand, hop_range, decay, -0.7, lamb, 0.3, ramp, soc_model)
    assert m.Norb == 2 * Nat
    assert np.max(np.abs(m.H - ref)) < 1e-13, np.max(np.abs(m.H - ref))
    assert np.allclose(m.H, m.H.conj().T, atol=0, rtol=0)


def test_peptide_defaults_are_the_alpha_helix(tmp_path):
    """pep_twist 100 deg, rise 1.5, hop_range 1, decay 1, radial SOC, no ramp by default."""
    Nat, R = 7, 2.3
    (tmp_path / "input.dat").write_text(COMMON + f"hamiltonian = peptide\nN_sites = {Nat}\nhel_radius = {R}\n"
                                                 "lamb = 0.01\n")
    m = qb.Model.load(str(tmp_path))
    ref = peptide_h(Nat, 100.0, 1.5, R, 1, 1, 1.0, -0.7, 0.01, 0.3, 0.0, "radial")
    assert np.max(np.abs(m.H - ref)) < 1e-13
