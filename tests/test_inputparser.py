"""goSPL YAML input subset (gospl/tools/inputparser.py) read by Model(filename)."""
import numpy as np
import pytest

from gospl_b200.inputparser import parse_bc, read_input

YML = """name: incising-like
domain:
    npdata: ['{mesh}','v','c','z']
    flowdir: 3
    bc: '0f01'
    nodep: False
    seadepo: False
time:
    start: 0.
    end: 300.
    tout: 300
    dt: 100.
spl:
    K: 4.0e-6
    d: 0.
    m: 0.5
    G: 0.
diffusion:
    hillslopeKa: 0.01
    hillslopeKm: 0.2
sea:
    position: -100.
climate:
  - start: 0.
    uniform: 1
tectonics:
  - start: 0.
    end: 300.
    upsub: ['{mesh}', 'u']
"""


def _write(tmp_path, text):
    rng = np.random.default_rng(3)
    v = rng.random((10, 3))
    c = np.array([[0, 1, 2], [2, 3, 4]], np.int32)
    np.savez(tmp_path / "m.npz", v=v, c=c, z=rng.random(10), u=np.full(10, 1e-3))
    y = tmp_path / "in.yml"
    y.write_text(text.format(mesh=str(tmp_path / "m")))
    return y, v


def test_reads_the_path_keys(tmp_path):
    y, v = _write(tmp_path, YML)
    coords, cells, elev, p = read_input(str(y))
    assert np.array_equal(coords, v) and cells.shape == (2, 3) and elev.shape == (10,)
    assert p["flowDir"] == 3 and p["bc"] == "ofof"
    assert (p["tStart"], p["tEnd"], p["dt"], p["tout"]) == (0.0, 300.0, 100.0, 300.0)
    assert (p["K"], p["d"], p["m"]) == (4.0e-6, 0.0, 0.5)
    assert (p["Cda"], p["Cdm"], p["oFill"], p["sealevel"]) == (0.01, 0.2, -6000.0, -100.0)
    assert np.all(p["rain"] == 1.0) and np.allclose(p["upsub"], 1e-3)
    assert (p["nodep"], p["seadepo"], p["nlPitVolume"], p["nlPitDepth"]) == (False, False, 1.0e9, 100.0)
    # lake diffusion keys of the diffusion section (inputparser.py:546-593)
    assert (p["nlPitK"], p["pitInletBias"], p["marineSolver"], p["picardSub"], p["picardIts"]) == \
        (10.0, 0.10, "ts", 10, 2)
    y, _ = _write(tmp_path, YML.replace("    hillslopeKm: 0.2\n", "    hillslopeKm: 0.2\n    nonlinKm: 4.0\n"
                                        "    marineSolver: Picard\n    picardSub: 3\n"))
    q = read_input(str(y))[3]
    assert (q["nlPitK"], q["marineSolver"], q["picardSub"]) == (4.0, "picard", 3)


def test_marine_deposition_needs_the_picard_solver(tmp_path):
    """goSPL's default (nodep False, seadepo True) also runs marine deposition
    with its adaptive TS solve of the marine diffusion, which this library
    does not build: the input must choose marineSolver picard (any Gmar) or
    switch marine deposition off."""
    y, _ = _write(tmp_path, YML.replace("    seadepo: False\n", ""))
    with pytest.raises(ValueError, match="seadepo"):
        read_input(str(y))
    y, _ = _write(tmp_path, YML.replace("    seadepo: False\n", "").replace(
        "    hillslopeKa: 0.01\n", "    hillslopeKa: 0.01\n    marineSolver: picard\n    Gmar: 0.5\n"))
    _, _, _, p = read_input(str(y))
    assert (p["seadepo"], p["marineSolver"], p["Gmar"]) == (True, "picard", 0.5)
    y, _ = _write(tmp_path, YML.replace("    nodep: False\n    seadepo: False\n", "    nodep: True\n"))
    assert read_input(str(y))[3]["nodep"] is True


def test_defaults_and_errors(tmp_path):
    y, _ = _write(tmp_path, YML.replace("    G: 0.\n", "    G: 1.\n"))
    assert read_input(str(y))[3]["G"] == 1.0
    y, _ = _write(tmp_path, YML.replace("    end: 300.\n    tout", "    end: -1.\n    tout"))
    with pytest.raises(ValueError):
        read_input(str(y))
    with pytest.raises(ValueError):
        parse_bc("oox")
    with pytest.raises(ValueError):
        parse_bc("cooo")
    assert parse_bc("0101") == "ofof"
    y, _ = _write(tmp_path, YML.replace("spl:\n    K: 4.0e-6\n    d: 0.\n    m: 0.5\n    G: 0.\n", ""))
    _, _, _, p = read_input(str(y))
    assert (p["K"], p["d"], p["m"]) == (1.0e-12, 0.0, 0.5)


def test_output_and_restart_keys(tmp_path):
    """time.tout clamped to [dt, end - start], time.rstep, the output section
    (inputparser.py:404-429, 2096-2117)."""
    y, _ = _write(tmp_path, YML)
    p = read_input(str(y))[3]
    assert (p["outputDir"], p["makedir"], p["compression"], p["rStep"]) == ("output", False, "gzip", 0)
    assert p["finput"] == str(y)
    y, _ = _write(tmp_path, YML.replace("    tout: 300\n", "    tout: 900\n    rstep: 2\n")
                  + "output:\n    dir: run\n    makedir: True\n    compression: none\n")
    p = read_input(str(y))[3]
    assert (p["tout"], p["rStep"], p["outputDir"], p["compression"]) == (300.0, 2, "run", "none")
    assert p["makedir"] is False          # a restart reuses the directory
    y, _ = _write(tmp_path, YML.replace("    tout: 300\n", "    tout: 10\n"))
    assert read_input(str(y))[3]["tout"] == 100.0
