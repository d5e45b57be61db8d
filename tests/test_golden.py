"""The oracle against the golden vectors derived from the reference's tables
and closed-form routines (tests/golden/make_golden.py)."""
import json
import os

import numpy as np

import oracle

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def load(name):
    return json.load(open(os.path.join(G, name)))


def test_tea_and_lcg_streams():
    for c in load('sampler.json'):
        seed = oracle.tea(oracle.tea(c['px'], c['py']), oracle.tea(c['sample'], c['dim']))
        assert seed == c['seed']
        s = oracle.sampler_stream(c['px'], c['py'], c['sample'], c['dim'], len(c['stream']))
        assert np.array_equal(s, np.array(c['stream'], np.float32))


def test_cie_y_integral():
    g = load('cie_5nm.json')
    assert oracle.cie_y_integral() == np.float32(g['y_integral'])


def test_spd_eval():
    g = load('cie_5nm.json')
    for c in load('spd_eval.json'):
        tab = np.array(g['y'] if c['table'] == 'y' else g['d65'], np.float32)
        v = oracle.lib().oracle_spd_eval(tab.ctypes.data_as(__import__('ctypes').c_void_p), 94, c['lambda'])
        assert abs(v - c['value']) <= 1e-6 * max(1.0, abs(c['value'])), c


def test_hero_wavelengths():
    for c in load('wavelengths.json'):
        lam, pdf = oracle.wavelengths(c['n'], c['u'])
        np.testing.assert_allclose(lam, c['lambda'], rtol=2e-5)
        np.testing.assert_allclose(pdf, c['pdf'], rtol=2e-4)
        assert np.all((lam >= 359.9) & (lam <= 830.1))


def test_linear_srgb_of_constant_spectrum():
    # A constant spectrum integrates to the equal-energy white: Y = 1 for
    # uniform wavelength sampling, when averaged over many samples.
    acc = np.zeros(3)
    n = 4000
    for i in range(n):
        lam, pdf = oracle.wavelengths(4, (i + 0.5) / n)
        acc += oracle.linear_srgb(lam, pdf, np.ones(4, np.float32))
    acc /= n
    y = 0.212671 * acc[0] + 0.715160 * acc[1] + 0.072169 * acc[2]
    # The reference SPD spacing (471 / 94 nm) and trapezoid integral leave ~0.2 %.
    assert abs(y - 1.0) < 5e-3
