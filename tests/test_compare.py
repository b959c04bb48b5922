"""The diagnostics comparison tool (CPU): a synthetic reference curve in the external
DNS file's format (t E eps enstrophy, whitespace) against a CSV in the run driver's format."""
import json

import numpy as np

from spectral_solver_b200 import compare


def test_compare_reports_gaps_and_peaks(tmp_path, capsys):
    t = np.linspace(0.0, 20.0, 2001)
    eps = 0.0005 + 0.012 * np.exp(-((t - 9.0) / 2.0) ** 2)
    E = 0.125 - np.cumsum(eps) * (t[1] - t[0])
    ref = tmp_path / "ref.dat"
    np.savetxt(ref, np.column_stack([t, E, eps, eps * 800.0]))
    ts = np.arange(0.0, 20.0001, 1.0)
    ours = tmp_path / "ours.csv"
    e_ours = np.interp(ts, t, E) + 1e-4
    d_ours = np.interp(ts, t, eps)
    with open(ours, "w") as f:
        f.write("t,kinetic_energy,dissipation,enstrophy,max_spectral_divergence,max_velocity,dt,cfl,main_dt,main_cfl\n")
        for a, b, c in zip(ts, e_ours, d_ours):
            f.write(f"{a},{b},{c},{c * 800.0},0,1,0,0,0,0\n")
    aligned = tmp_path / "aligned.csv"
    assert compare.main(["--ours", str(ours), "--reference", str(ref), "--aligned", str(aligned)]) == 0
    rep = json.loads(capsys.readouterr().out)
    assert abs(rep["kinetic_energy"]["max_abs"] - 1e-4) < 1e-9
    assert rep["dissipation"]["max_abs"] < 1e-12
    assert rep["peak_dissipation"]["ours"][0] == 9.0 and abs(rep["peak_dissipation"]["reference"][0] - 9.0) < 1e-9
    assert rep["points"] == 21
    assert np.loadtxt(aligned, delimiter=",", skiprows=1).shape == (21, 7)
