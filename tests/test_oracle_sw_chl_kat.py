"""The oracle's chlorophyll shortwave (Manizza 2005 opacities, the N-band
split and the N-band penetration profile) against the reference's
known-answer tests (tests/test_ocean_sw_chl.F90), re-expressed on the oracle
(the Fortran tests cannot run here: no Fortran compiler).

Bottom-up like the reference: level 1 is the bed, nz the surface.  Checked
quantities and tolerances are the reference tests' own:
  opacities kappa_n = a_n + b_n chl^p_n at chl = 0.1, 1, 10 to 1e-14, a + b
      at chl = 1, a fill value floored at 1e-4, the land opacity 10 in every
      band, opacity growing with chlorophyll (test_kappa_values, :150-215);
  on 10 layers of 10 m with no tracer, one band at a time (kappa 0.05, 0.02,
      0.011 m^-1): layer k takes e^{-kappa z_top} - e^{-kappa z_bot}, the bed
      layer everything below its top, the column all of it, to 1e-13; three
      chlorophyll bands at chl = 0.5 with the default 0.21 / 0.21 / 0.58
      split: the same with the 3-band transmission, the bed layer the whole
      remainder, and a top layer unlike the two-band Jerlov I profile
      (test_column_absorption, :261-340);
  the band split: 0.21 / 0.21 / 0.58 of the shortwave at blue_frac 0.5,
      0.126 / 0.294 / 0.58 at 0.3, the infrared shared evenly over bands 3..5
      and the bands summing to 1 (test_band_split, :346-372).
A band "alone" is expressed here by giving all three bands its opacity: the
fractions sum to one, so the N-band transmission is that band's.
"""
import ctypes
import math

import numpy as np

from roundabout_b200.config import default_config

A1, B1, P1 = 0.0232, 0.074, 0.674
A2, B2, P2 = 0.225, 0.037, 0.629
K3 = 2.86
R2, ZETA1, ZETA2 = 0.58, 0.35, 23.0
CHL_FLOOR = 1.0e-4


def kappa_ref(n, chl):
    return (A1 + B1 * chl ** P1, A2 + B2 * chl ** P2, K3)[n]


def chl_cfg(**kw):
    c = default_config()
    c.sw_chl = 1
    c.sw_pen_frac = 1.0
    c.sw_nbands = 3
    c.sw_blue_frac = 0.5
    for n, v in enumerate((A1, B1, A2, B2, K3, 0.0)):
        c.sw_opacity_coef[n] = v
    for n, v in enumerate((P1, P2, 0.0)):
        c.sw_chl_power[n] = v
    c.sw_opacity_land = 10.0
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def band_frac(oracle, n, nb, blue):
    L = oracle.lib()
    L.vpo_sw_band_frac.restype = ctypes.c_double
    L.vpo_sw_band_frac.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    return L.vpo_sw_band_frac(n, nb, blue)


def test_opacities_at_the_reference_chlorophylls(oracle):
    chls = (0.1, 1.0, 10.0)
    st = oracle.OracleState(5, 3, 2, 2)
    for m, chl in enumerate(chls):
        st.sw_chl[m, :] = chl
    st.sw_chl[3, :] = -1.0e34          # a fill value
    st.wet[4, :] = 0.0                 # land
    st.call("vpo_sw_chl_kappa", chl_cfg())
    kap = st.sw_kappa[:, 1, :]
    for m, chl in enumerate(chls):
        for n in range(3):
            assert abs(kap[m, n] - kappa_ref(n, chl)) < 1.0e-14, (m, n)
    assert abs(kap[1, 0] - (A1 + B1)) < 1.0e-14 and abs(kap[1, 1] - (A2 + B2)) < 1.0e-14
    for n in range(3):
        assert abs(kap[3, n] - kappa_ref(n, CHL_FLOOR)) < 1.0e-14, n
        assert kap[4, n] == 10.0, n
    assert kap[2, 0] > kap[1, 0] > kap[0, 0] and kap[2, 1] > kap[0, 1]


NZ, DZ, QSW, DT = 10, 10.0, 300.0, 1800.0


def absorbed_fractions(oracle, kappas):
    """The share of the shortwave each layer keeps, the surface lump the
    deposit left in the top layer put back (deposit_column, :221-259)."""
    c = chl_cfg()
    st = oracle.OracleState(6, 4, NZ, 2)
    st.h[...] = DZ
    st.q_heat[...] = QSW
    for n, k in enumerate(kappas):
        st.sw_kappa[:, :, n] = k
    st.call("vpo_sw_penetration", c, DT)
    got = st.tracers[c.idx_temperature][3, 2, :] * DZ / (DT / (c.rho0 * c.cp) * QSW)
    got[NZ - 1] += 1.0
    return got


def trans(d, kap, frac):
    return sum(f * math.exp(-k * d) for k, f in zip(kap, frac))


def test_one_band_alone_is_absorbed_layer_by_layer(oracle):
    for kb in (0.05, 0.02, 0.011):
        got = absorbed_fractions(oracle, (kb, kb, kb))
        for k in range(1, NZ + 1):
            ztop = (NZ - k) * DZ
            want = math.exp(-kb * ztop) - (math.exp(-kb * (ztop + DZ)) if k > 1 else 0.0)
            assert abs(got[k - 1] - want) < 1.0e-13, (kb, k)
        assert abs(got.sum() - 1.0) < 1.0e-13, kb


def test_three_chlorophyll_bands_absorbed_and_conserved(oracle):
    kap = [kappa_ref(n, 0.5) for n in range(3)]
    frac = (0.21, 0.21, 0.58)
    got = absorbed_fractions(oracle, kap)
    for k in range(1, NZ + 1):
        ztop = (NZ - k) * DZ
        want = trans(ztop, kap, frac) - (trans(ztop + DZ, kap, frac) if k > 1 else 0.0)
        assert abs(got[k - 1] - want) < 1.0e-13, k
    assert abs(got.sum() - 1.0) < 1.0e-13
    assert got[0] > 0.0 and abs(got[0] - trans((NZ - 1) * DZ, kap, frac)) < 1.0e-13
    two_band_top = R2 * (1.0 - math.exp(-DZ / ZETA1)) + (1.0 - R2) * (1.0 - math.exp(-DZ / ZETA2))
    assert abs(got[NZ - 1] - two_band_top) > 1.0e-3


def test_band_split(oracle):
    SW = 400.0
    f3 = [band_frac(oracle, n, 3, 0.5) for n in (1, 2, 3)]
    assert all(abs(f * SW - w * SW) < 1.0e-13 for f, w in zip(f3, (0.21, 0.21, 0.58)))
    assert abs(sum(f3) * SW - SW) < 1.0e-13
    f3b = [band_frac(oracle, n, 3, 0.3) for n in (1, 2, 3)]
    assert all(abs(f - w) < 1.0e-15 for f, w in zip(f3b, (0.126, 0.294, 0.58)))
    f5 = [band_frac(oracle, n, 5, 0.5) for n in range(1, 6)]
    assert abs(f5[2] - 0.58 / 3.0) < 1.0e-15 and abs(f5[3] - f5[2]) < 1.0e-15 and abs(f5[4] - f5[2]) < 1.0e-15
    assert abs(sum(f5) - 1.0) < 1.0e-14
