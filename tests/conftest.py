"""Shared test setup: import paths, the `gpu` marker, golden-fixture loaders."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "softx-d-15-00085_b200")
for p in (PKG, os.path.join(REPO, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

from blaze import types as T  # noqa: E402

GOLDEN = os.path.join(REPO, "tests", "golden")
# the reference tree (only the CPU tests that compile or parse it read it):
# $BLAZE_REFERENCE, else a directory "reference" beside the repository
REFERENCE = os.environ.get("BLAZE_REFERENCE", os.path.join(os.path.dirname(REPO), "reference"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built library")


class Golden:
    """A golden fixture: boundary structs + initial state + oracle-A checkpoints."""

    def __init__(self, name):
        self.name = name
        self.z = np.load(os.path.join(GOLDEN, name + ".npz"))
        z = self.z
        self.n_w, self.n_p, self.n_d = int(z["n_w"]), int(z["n_p"]), int(z["n_d"])
        self.cyl_rot = bool(int(z["cyl_rot"]))
        self.wobj = (T.WOBJ * 8).from_buffer_copy(z["wobj"].tobytes())
        self.pobj = (T.POBJ * 8).from_buffer_copy(z["pobj"].tobytes())
        self.dobj = (T.DOBJ * 32).from_buffer_copy(z["dobj"].tobytes())
        self.sim_info = T.SimulationInfo.from_buffer_copy(z["sim_info"].tobytes())
        self.sim_info.Num_ParticlesPerObject = None
        self.n = self.sim_info.Num_Particles
        self.checkpoints = sorted(int(k[1:].split("_")[0]) for k in z.files
                                  if k.startswith("s") and k.endswith("_pos"))

    def init(self):
        z = self.z
        out = dict(pos=z["init_pos"], vel=z["init_vel"], avel=z["init_avel"],
                   type=z["init_type"], pid=z["init_pid"])
        if "init_quat" in z.files:
            out["quat"] = z["init_quat"]
        return out

    def at(self, k):
        z = self.z
        keys = ["pos", "vel", "avel", "type", "pid", "f_pp", "t_pp", "f_wall", "t_wall",
                "f_lift", "t_lift", "nn", "list"]
        if "s%d_quat" % k in z.files:
            keys.append("quat")
        return {key: z["s%d_%s" % (k, key)] for key in keys}


GOLDEN_NAMES = ["silo_sph90", "mill_sph30"]
POLY_GOLDEN_NAMES = ["box_poly", "drum_poly", "lifter_poly"]


@pytest.fixture(params=GOLDEN_NAMES)
def golden(request):
    return Golden(request.param)


@pytest.fixture(params=POLY_GOLDEN_NAMES)
def golden_poly(request):
    return Golden(request.param)


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
