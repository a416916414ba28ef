"""The benchmark's reference arm builds the same workload as the eup arm without the
product library: its plain-number description, the oracle's voxeliser and the oracle's
seeded initial state are held equal to euplectella_hpc_b200.workloads here (CPU only)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ROOT)
    import bench as B
    return B


@pytest.mark.parametrize("name", ["cylinder", "shell"])
def test_spec_matches_workload(eup, bench, name):
    from euplectella_hpc_b200 import workloads
    spec = bench.SPECS[name]
    wl = workloads.reticular_shell_channel() if name == "shell" else workloads.cylinder_channel()
    c = wl.cfg
    assert spec["name"] == wl.name
    assert tuple(spec["lattice"]) == (c.lx, c.ly, c.lz)
    assert tuple(spec["bc"]) == tuple(c.bc)
    assert bench.spec_svisc(spec) == c.svisc
    assert spec["u_in"] == c.u_inflow and c.u0 == 0.0 and c.u00 == 0.0
    assert spec["seed"] == wl.seed
    g = wl.geometry
    b = spec["body"]
    if name == "shell":
        assert (g.x0, g.length, g.yc, g.zc, g.outer_d, g.strut_d, g.pitch, g.seed) == (
            b["x0"], b["length"], b["yc"], b["zc"], b["outer_d"], b["strut_d"], b["pitch"], b["seed"])
    else:
        assert (g.xc, g.yc, g.radius) == (b["xc"], b["yc"], b["r"])
    # full-size mask from the oracle's voxeliser, bit for bit the product's
    obs, _ = bench.reference_input(dict(spec, lattice=(4, 4, 4)), np.float32)  # warms the oracle library
    from oracle import oracle as O
    lx, ly, lz = spec["lattice"]
    if name == "shell":
        obs = O.voxelise_shell(lx, ly, lz, b["x0"], b["length"], b["yc"], b["zc"], b["outer_d"], b["strut_d"],
                               b["pitch"], b["seed"])
    else:
        obs = O.voxelise_cylinder_z(lx, ly, lz, b["xc"], b["yc"], b["r"])
    assert np.array_equal(obs, wl.obs)
    # initial state: the oracle's seeded equilibrium equals the product's (cylinder at full size;
    # the shell's 17 GB state at a reduced lattice with the same seed)
    if name == "cylinder":
        _, state = bench.reference_input(spec, np.float32)
        assert np.array_equal(state, wl.initial_state(np.float32))
    else:
        small = eup.init_equilibrium(40, 24, 16, spec["u_in"], bench.PERTURBATION, spec["seed"], np.float32)
        assert np.array_equal(O.init_perturbed(40, 24, 16, spec["u_in"], bench.PERTURBATION, spec["seed"]), small)


def test_reference_arm_loads_no_product_library(tmp_path):
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'cylinder', "
            "'--steps', '2', '--warmup', '1']; runpy.run_path('bench.py', run_name='__main__')")
    probe = ("import atexit\n"
             "def _maps():\n"
             "    libs = sorted({l.split()[-1] for l in open('/proc/self/maps') if l.rstrip().endswith('.so')})\n"
             "    print('MAPPED ' + ' '.join(libs))\n"
             "atexit.register(_maps)\n")
    r = subprocess.run([sys.executable, "-c", probe + code], cwd=ROOT, capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, OMP_NUM_THREADS="2"))
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    line = json.loads([x for x in lines if x.startswith("{")][-1])
    mapped = [x for x in lines if x.startswith("MAPPED")][-1]
    assert "libeup" not in mapped and "liborc.so" in mapped
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["workload"] == "cylinder_256x128x64_re100"
    assert line["config"]["solid_voxels"] == 64 * 317
