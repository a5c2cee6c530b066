"""The command line's option grammar and input loading (floodca_b200.cli),
on the CPU: the reference's `--key value` / `--key=value` / `--config`
forms, its defaults, the rain file with lambda and the warm start as the
reference's CLIs load them (src/common/grid.c:239-268, main_cuda.c:39-55)."""
import numpy as np
import pytest

from floodca_b200 import cli, synth
from floodca_b200.sim import RunParams


def test_parse_reference_grammar(tmp_path):
    ini = tmp_path / "run.ini"
    ini.write_text("# comment\nalpha = 0.4\nneigh = 8\nhyeto = uniform\n")
    o = cli.parse(["--grid", "G", "--config", str(ini), "--tsim=7200", "--U", "2",
                   "--boundary", "closed", "--threads", "16", "--no-output",
                   "--edges", "0100", "--rain_end", "3600", "--inflow_cell", "0,5",
                   "--inflow_peak", "500", "--precision", "f64"])
    assert o.grid == "G" and o.no_output and o.precision == "f64" and o.inflow_rc == (0, 5)
    assert o.params == dict(alpha=0.4, K=8, hyeto="uniform", T_sim=7200.0, U=2,
                            boundary="closed", edges=(0, 1, 0, 0), rain_end=3600.0,
                            inflow_peak=500.0)
    with pytest.raises(cli.UsageError):
        cli.parse(["--tsim", "10"])                  # no grid
    with pytest.raises(cli.UsageError):
        cli.parse(["--grid", "G", "--edges", "01"])
    with pytest.raises(cli.UsageError):
        cli.parse(["--grid", "G", "--forcing", "f.csv"])


def test_inputs_rain_lambda_warmstart(tmp_path):
    d = synth.make_terrain(synth.TerrainSpec(12, 9, seed=2))
    d.Rday = np.full(d.shape, 0.1, np.float32)
    synth.write_grid_dir(d, tmp_path / "g")
    rain = np.linspace(0, 0.3, 12 * 9, dtype=np.float32).reshape(12, 9)
    rain.tofile(tmp_path / "rain.bin")
    warm = np.full((12, 9), 0.05, np.float32)
    warm.tofile(tmp_path / "warm.bin")

    dom, p = cli.inputs(cli.parse(["--grid", str(tmp_path / "g"), "--lambda", "2"]))
    # without a rain file, lambda leaves the grid's Rday alone (grid.c:256-268)
    assert p.lambda_ == 1.0 and np.array_equal(dom.Rday, d.Rday)
    assert p == RunParams()                       # the reference defaults otherwise

    dom, p = cli.inputs(cli.parse(["--grid", str(tmp_path / "g"), "--rain",
                                   str(tmp_path / "rain.bin"), "--lambda", "2",
                                   "--warmstart", str(tmp_path / "warm.bin"),
                                   "--inflow_cell", "3,4"]))
    assert p.lambda_ == 2.0 and np.array_equal(dom.Rday, rain)
    assert np.array_equal(dom.h, warm) and np.array_equal(dom.hmax, warm)
    assert p.inflow_cell == 3 * 9 + 4
    with pytest.raises(cli.UsageError):
        cli.inputs(cli.parse(["--grid", str(tmp_path / "g"), "--inflow_cell", "12,0"]))
