"""The reference's output files (pops.dat, _states_<t>.dat, correlation and spectrum text files)
written from the ensemble's observables: layout and values parsed back and compared with the
getters, numpy and the reference's formatting rules."""
import struct

import numpy as np
import pytest

from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu


def _prop(pop_every=1, steps=20):
    import dynaquant_b200 as dq
    from dynaquant_b200 import systems
    c = G.CHAIN
    s = systems.chain(256, c["J"])
    p = dq.Propagator(s.n, m=c["m"], n_traj=4, dt=c["dt"], noise=dq.NOISE_OU, sigma_static=c["sigma_static"],
                      seed=c["seed"], dot=1, pop_every=pop_every, max_steps=steps, precision=dq.PREC_FP64)
    p.set_system(s)
    p.set_noise_params(np.full(s.n, c["sigma"]), np.full(s.n, c["tau"]))
    psi0 = np.zeros(s.n, complex)
    psi0[128] = 1.0
    p.set_initial_state(psi0)
    p.run(steps)
    return p, s


def _parse_text_pops(path, n):
    lines = open(path).read().splitlines()
    head = {ln.split()[0]: ln.split()[1] for ln in lines[:4]}
    steps, vals, k = [], [], 4
    while k < len(lines):
        assert lines[k].startswith("STEP ")
        steps.append(int(lines[k].split()[1]))
        row = []
        for i in range(n):
            ln = lines[k + 1 + i]
            assert len(ln) == 25 + len(f" ({i})") and ln.endswith(f" ({i})")
            row.append(float(ln[:25]))
        vals.append(row)
        k += n + 1
    return head, steps, np.array(vals)


def test_pops_text_and_continuation(tmp_path):
    p, s = _prop(pop_every=2, steps=20)
    path = tmp_path / "pops.dat"
    p.write_populations(path)
    head, steps, vals = _parse_text_pops(path, s.n)
    assert head == {"numsims": "4", "dt": "1", "totalsteps": "20", "numprintedsites": str(s.n)}
    assert steps == list(range(2, 21, 2))
    sums = p.populations()[1:] * 4
    assert np.abs(vals - sums).max() <= 1e-15 * np.abs(sums).max()
    assert "%25.17g (%d)" % (sums[0, 0], 0) == open(path).read().splitlines()[5]
    # a second batch of runs adds into the same file
    p.write_populations(path, continuation=True)
    head2, _, vals2 = _parse_text_pops(path, s.n)
    assert head2["numsims"] == "8"
    assert np.abs(vals2 - 2 * sums).max() <= 1e-14 * np.abs(sums).max()
    assert not (tmp_path / "temp_pops.dat").exists()
    p.close()


def test_pops_binary(tmp_path):
    p, s = _prop()
    path = tmp_path / "pops.bin"
    p.write_populations(path, binary=True)
    raw = open(path, "rb").read()
    numsims, dt, steps, sites = struct.unpack("<idii", raw[:20])
    assert (numsims, dt, steps, sites) == (4, 1.0, 20, s.n)
    vals = np.frombuffer(raw[20:], dtype="<f8").reshape(20, s.n)
    # the getter's 1/n_traj scaling is exact except in the subnormal range
    assert np.allclose(vals, p.populations()[1:] * 4, rtol=1e-15, atol=1e-300)
    p.write_populations(path, binary=True, continuation=True)
    raw2 = open(path, "rb").read()
    assert struct.unpack("<i", raw2[:4])[0] == 8
    p.close()


def test_states_file(tmp_path):
    p, s = _prop()
    p.write_states(tmp_path)
    f = tmp_path / "_states_20.dat"
    raw = open(f, "rb").read()
    stamp, n, runs = struct.unpack("<fii", raw[:12])
    assert (stamp, n, runs) == (20.0, s.n, 4)
    st = np.frombuffer(raw[12:], dtype="<c16").reshape(4, s.n)
    assert np.array_equal(st, p.states())
    p.close()


def test_spectrum_files(tmp_path):
    p, s = _prop(steps=20)
    corr = p.correlation()
    scaling = 3.7
    p.write_spectrum(tmp_path / "absCorrFunc.dat", tmp_path / "absorption.dat", scaling)
    sc = float(np.float32(scaling))
    cl = open(tmp_path / "absCorrFunc.dat").read().splitlines()
    assert cl[0] == "{timestep #} {timestamp fs} {M(t) real imag}: "
    for i in (0, 7, 20):
        row = cl[1 + i]
        assert row == "%6d%14g%14g%14g" % (i, i * 1.0, corr[i].real * sc, corr[i].imag * sc)
    T = 20
    spec = np.fft.ifft(corr) * len(corr)          # length T + 1, unnormalised inverse DFT
    sl = open(tmp_path / "absorption.dat").read().splitlines()
    assert sl[0] == "{k #} {freq rev/fs} {freq cm^-1} {Transform real imag}: "
    f = np.float32(sc) / np.float32(T)
    for fid in range(T + 1):
        k = fid - T if fid > T // 2 else fid
        parts = sl[1 + fid].split()
        assert int(parts[0]) == k
        assert float(parts[1]) == pytest.approx(k / (T * 1.0), rel=1e-5, abs=1e-12)
        assert float(parts[2]) == pytest.approx(k / (299792458. * 100 * 1e-15) / T, rel=1e-5, abs=1e-9)
        assert float(parts[3]) == pytest.approx(spec[fid].real * float(f), rel=1e-5, abs=1e-9)
        assert float(parts[4]) == pytest.approx(spec[fid].imag * float(f), rel=1e-5, abs=1e-9)
    p.close()


def test_line_dressing(tmp_path):
    """Gaussian line-shape dressing: M(k) exp(-(dt (k+1) / sigma)^2 / 2) for k < steps before the
    transforms (the reference's offset by one), in the files and in dq_get_spectrum."""
    p, s = _prop(steps=20)
    corr = p.correlation()
    plain = p.spectrum(32)
    sigma = 7.0
    p.set_line_dressing(sigma)
    k = np.arange(21)
    g = np.where(k < 20, np.exp(-0.5 * ((k + 1) * 1.0 / sigma) ** 2), 1.0)
    dressed = corr * g
    spec = p.spectrum(32)
    ref = np.fft.ifft(np.concatenate([dressed, np.zeros(11)])) * 32
    assert np.abs(spec - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(spec - plain).max() > 1e-6
    p.write_spectrum(tmp_path / "c.dat", tmp_path / "s.dat", 1.0)
    row = open(tmp_path / "c.dat").read().splitlines()[1 + 5].split()
    assert float(row[2]) == pytest.approx(dressed[5].real, rel=1e-5, abs=1e-12)
    p.set_line_dressing(0.0)
    assert np.abs(p.spectrum(32) - plain).max() == 0.0
    import dynaquant_b200 as dq
    with pytest.raises(dq.DQError):
        p.set_line_dressing(-1.0)
    p.close()
