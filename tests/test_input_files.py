"""The readers of the reference's input files (dynaquant_b200.io) on small files in its formats."""
import numpy as np
import pytest

from dynaquant_b200 import io


def test_hamiltonian_general_and_symmetric(tmp_path):
    g = tmp_path / "hg.dat"
    g.write_text("%%MatrixMarket matrix coordinate real general\nBASE_ONE\n3 3 5\n"
                 "1 1 10.0\n1 2 -5.0\n2 1 -5.0\n2 2 20.0\n3 3 30.0\n")
    n, rp, col, val = io.read_hamiltonian(g)
    dense = np.zeros((n, n))
    for i in range(n):
        for p in range(rp[i], rp[i + 1]):
            dense[i, col[p]] += val[p]
    assert np.allclose(dense, [[10, -5, 0], [-5, 20, 0], [0, 0, 30]])
    s = tmp_path / "hs.dat"
    # lower triangle used and mirrored; an entry above the diagonal is ignored as cuSPARSE does
    s.write_text("%%MatrixMarket matrix coordinate real symmetric\nBASE_ZERO\n3 3 5\n"
                 "0 0 1.0\n1 0 2.0\n2 1 3.0\n0 2 99.0\n2 2 4.0\n")
    n, rp, col, val = io.read_hamiltonian(s)
    dense = np.zeros((n, n))
    for i in range(n):
        for p in range(rp[i], rp[i + 1]):
            dense[i, col[p]] += val[p]
    assert np.allclose(dense, [[1, 2, 0], [2, 0, 3], [0, 3, 4]])
    with pytest.raises(ValueError):
        bad = tmp_path / "hb.dat"
        bad.write_text("%%MatrixMarket matrix coordinate real general\nBASE_ZERO\n2 2 1\n5 0 1.0\n")
        io.read_hamiltonian(bad)


def test_parameter_and_state_files(tmp_path):
    ka = tmp_path / "ka.dat"
    ka.write_text("100 200\n50 250\n")
    sigma, tau = io.read_ka_params(ka, 2)
    assert np.allclose(sigma, [200, 250]) and np.allclose(tau, [100, 50])
    hsr = tmp_path / "hsr.dat"
    hsr.write_text("10\n20\n30\n")
    assert np.allclose(io.read_hsr_stddev(hsr, 3), [10, 20, 30])
    st = tmp_path / "init.dat"
    st.write_text("BASE_ZERO\nsome comment\n1 3.0\n2 4.0\nEND\n3 7.0\n")
    psi = io.read_initial_state(st, 4)
    assert np.allclose(psi, [0, 0.6, 0.8, 0])
    dip = tmp_path / "dips.dat"
    dip.write_text("   -0.0554    0.8188    0.5714\n   -0.2824   -0.7705    0.5714\n")
    v = io.read_vectors3(dip)
    assert v.shape == (2, 3) and v[1, 1] == -0.7705


def test_spectral_density_file(tmp_path, oracle):
    f = tmp_path / "specd.dat"
    f.write_text("8.135709639 2\n8.135709639\t2.082740586\n16.27141928\t7.325068785\n")
    d_omega, om, J = io.read_spectral_density(f)
    assert d_omega == 8.135709639 and len(om) == 2
    w, c = oracle.zz_coefficients(om, J, d_omega, 77.0)
    # the reference's log prints oscillator 0 as OmegaVal = 0.00153248, coeffVal = 8.74586
    assert float(f"{w[0]:.6g}") == 0.00153248 and float(f"{c[0]:.6g}") == 8.74586
