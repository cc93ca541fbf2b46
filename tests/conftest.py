import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    import numpy as np
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def golden_flags(g):
    """Control flags of a golden case (cases without picard entries ran with
    the reference's default f46 = 0, f47 = 10)."""
    return dict(f43=float(g["f43"]), f44=int(g["f44"]), f45=float(g["f45"]), f49=int(g["f49"]),
                n47=float(g["n47"]), f46=int(g.get("f46", 0)), f47=int(g.get("f47", 10)))


def golden_ioflow(g):
    """Inflow / outflow flags of an io golden case (None for a closed box;
    the wave cases' faces, owned by iowave, at the reference's defaults)."""
    if "wave_wgen" in g:
        return dict(inflow=1, outflow=1)
    if "io_f50" not in g:
        return None
    ints = ("inflow", "outflow", "f50", "b77", "f64")
    return {k[3:]: (int(g[k]) if k[3:] in ints else float(g[k])) for k in g if k.startswith("io_")}


def golden_df(g):
    """(x45, body1, body2) of a direct-forcing golden case, else None."""
    if "x45" not in g:
        return None
    return int(g["x45"]), g["body1"], g["body2"]


def golden_wave(g):
    """(generation weights, beach weights, still water level, per-step
    targets, per-step ramps) of a wave-generator golden case, else None."""
    if "wave_wgen" not in g:
        return None
    return (g["wave_wgen"], g["wave_wbeach"], float(g["wave_phimean"]), g["step_wave_targets"],
            g["step_wave_ramp"])


def golden_sf(g):
    """The solid-forcing list (n, 4) of an sf golden case, else None."""
    return g["sf"] if "sf" in g else None


def body_field(x45, body1, body2):
    """The one body field the device stencils read: body1, or for X45 = 5
    min(solid, topo), which is > 0 exactly where both are."""
    import numpy as np
    return np.ascontiguousarray(np.minimum(body1, body2) if x45 == 5 else body1)


@pytest.fixture(scope="session")
def port_lib():
    """The C restatement oracle, built on demand (test infrastructure)."""
    import subprocess
    subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile")], check=True, cwd=ROOT)
    from oracle.bindings import PortOracle
    PortOracle.lib()
    return PortOracle


def velocity_at(g, t):
    """Stored velocity of a golden case at time t (the vortex cases scale the
    spatial field by cos(pi t / 3), as tests/golden/make_golden.py did)."""
    import numpy as np
    u, v, w = g["u"], g["v"], g["w"]
    if str(g["vel_scale"]) == "vortex":
        f = np.cos(np.pi * t / 3.0)
        u, v, w = u * f, v * f, w * f
    return np.ascontiguousarray(u), np.ascontiguousarray(v), np.ascontiguousarray(w)
