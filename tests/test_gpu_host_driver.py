"""The C++ host driver (dq_infile_run, the dq_propagate command) on input files
in the reference's formats, against the same run set up from Python through
the C ABI: the output files must be equal byte for byte."""
import os
import subprocess

import numpy as np
import pytest

import dynaquant_b200 as dq
from dynaquant_b200 import host, io, spectra, systems

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _write_system(d, n=96, seed=3):
    """A disordered chain as a symmetric BASE_ONE coordinate file (lower triangle),
    KA parameters, dipoles and positions."""
    rng = np.random.default_rng(seed)
    eps = rng.normal(0.0, 80.0, n)
    lines = ["%%MatrixMarket matrix coordinate real symmetric", "BASE_ONE"]
    ent = [(i + 1, i + 1, eps[i]) for i in range(n)] + [(i + 2, i + 1, -250.0 + 10 * rng.normal()) for i in range(n - 1)]
    lines.append(f"{n} {n} {len(ent)}")
    lines += [f"{i} {j} {v:.10f}" for i, j, v in ent]
    (d / "ham.dat").write_text("\n".join(lines) + "\n")
    (d / "ka.dat").write_text("".join(f"{60 + i % 7} {150 + 3 * (i % 5)}\n" for i in range(n)))
    mu = rng.normal(size=(n, 3))
    (d / "dips.dat").write_text("".join(f"{a:.6f} {b:.6f} {c:.6f}\n" for a, b, c in mu))
    R = np.stack([np.arange(n) * 8.0, np.zeros(n), np.zeros(n)], axis=1) + rng.normal(size=(n, 3))
    (d / "pos.dat").write_text("".join(f"{a:.6f} {b:.6f} {c:.6f}\n" for a, b, c in R))
    return n


def _python_prop(d, n, runs, steps, m, seed, sigma_static, traj0=0, pop_every=1):
    nn, rp, col, val = io.read_hamiltonian(d / "ham.dat")
    assert nn == n
    sigma, tau = io.read_ka_params(d / "ka.dat", n)
    p = dq.Propagator(n, m=m, n_traj=runs, dt=1.0, noise=dq.NOISE_OU, ka_substeps=2, sigma_static=sigma_static,
                      seed=seed, dot=dq.DOT_BILINEAR, norm=dq.NORM_REAL_ONLY, precision=dq.PREC_FP64,
                      pop_every=pop_every, max_steps=steps)
    p.set_hamiltonian_csr(rp, col, val)
    p.set_noise_params(sigma, tau)
    p.set_trajectory_offset(traj0)
    return p


INFILE = """! written by the test
dt = 1.0
totalsteps = {steps}
ensembleavgmode = ENS_AVG_MODE_FIRST
ensembleruns = {runs}
m = {m}
ka_substeps = 2
simtype = SIM_TYPE_KUBO_ANDERSON
ka_paramsfile = ka.dat
staticdis = 1
sigmastatdis = 60
writeoutpops = 1
printallpops = 1
writebinarypops = {binary}
writeoutstates = {states}
initstate = 40
hamfile = ham.dat
outfolder = out
seed = {seed}
{extra}
"""


@pytest.mark.parametrize("binary", [0, 1])
def test_driver_pops_equal_python_run_byte_for_byte(tmp_path, binary):
    n = _write_system(tmp_path)
    runs, steps, m, seed = 8, 30, 10, 17
    (tmp_path / "run.in").write_text(INFILE.format(steps=steps, runs=runs, m=m, binary=binary, states=10, seed=seed,
                                                   extra=""))
    host.run_infile(tmp_path / "run.in", base_dir=tmp_path)
    got = (tmp_path / "out" / "pops.dat").read_bytes()
    p = _python_prop(tmp_path, n, runs, steps, m, seed, 60.0)
    psi0 = np.zeros(n, complex)
    psi0[40] = 1.0
    p.set_initial_state(psi0)
    ref_dir = tmp_path / "py"
    ref_dir.mkdir()
    for k in range(3):
        p.run(10)
        p.write_states(str(ref_dir))
    p.write_populations(str(ref_dir / "pops.dat"), binary=bool(binary))
    assert got == (ref_dir / "pops.dat").read_bytes()
    st_host = sorted(f for f in os.listdir(tmp_path / "out") if f.startswith("_states_"))
    st_py = sorted(f for f in os.listdir(ref_dir) if f.startswith("_states_"))
    assert st_host == st_py and len(st_host) == 3
    for f in st_host:
        assert (tmp_path / "out" / f).read_bytes() == (ref_dir / f).read_bytes()
    p.close()


def test_driver_absorption_spectrum_equals_python_run(tmp_path):
    n = _write_system(tmp_path)
    runs, steps, m, seed = 4, 40, 10, 5
    (tmp_path / "run.in").write_text(INFILE.format(
        steps=steps, runs=runs, m=m, binary=0, states=0, seed=seed,
        extra="absorbspec = 1\ndipolefile = dips.dat\nlineshapedress = 1\ngausswidth = 30\nwriteoutpops = 0"))
    host.run_infile(tmp_path / "run.in", base_dir=tmp_path)
    mu = io.read_vectors3(tmp_path / "dips.dat")
    props, scal = [], []
    ref_dir = tmp_path / "py"
    ref_dir.mkdir()
    for d, (psi0, sc) in enumerate(spectra.absorption_directions(mu)):
        p = _python_prop(tmp_path, n, runs, steps, m, seed, 60.0, traj0=d * runs)
        p.set_initial_state(psi0)
        p.set_line_dressing(30.0)
        p.run(steps)
        p.write_spectrum(str(ref_dir / f"absCorrFuncDir{d}.dat"), str(ref_dir / f"absDir{d}.dat"), sc)
        props.append(p)
        scal.append(sc)
    spectra.write_spectrum_mean(props, scal, ref_dir / "absCorrFunc.dat", ref_dir / "absorption.dat")
    for f in ["absCorrFuncDir0.dat", "absDir2.dat", "absCorrFunc.dat", "absorption.dat"]:
        assert (tmp_path / "out" / f).read_bytes() == (ref_dir / f).read_bytes(), f
    assert not (tmp_path / "out" / "pops.dat").exists()
    for p in props:
        p.close()


def test_command_line_driver_runs_an_input_file(tmp_path):
    _write_system(tmp_path)
    (tmp_path / "run.in").write_text(INFILE.format(steps=12, runs=4, m=8, binary=0, states=0, seed=1,
                                                   extra="print_partic = 1"))
    exe = os.path.join(ROOT, "dynaquant_b200", "dq_propagate")
    r = subprocess.run([exe, "run.in"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    pops = (tmp_path / "out" / "pops.dat").read_text().splitlines()
    assert pops[0] == "numsims 4" and pops[2] == "totalsteps 12"
    ipr = (tmp_path / "invParticRat.dat").read_text().splitlines()
    assert ipr[0].startswith("#") and len(ipr) == 2 + 12
