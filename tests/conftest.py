import os
import sys

# expandable allocator segments (set before CUDA starts): the bounded-memory
# test of a nao 288 gradient frees and allocates tensors of tens of GB, which
# a segment-splitting cache fragments
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    import torch
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


class GoldenMol:
    """_atm/_bas/_env container rebuilt from a golden fixture."""

    def __init__(self, d):
        import numpy as np
        from ccsd_gpu_b200.gto.mole import Mole
        self._atm = d["atm"]
        self._bas = d["bas"]
        self._env = d["env"]
        self.cart = bool(d["cart"])
        self._c2s = d["c2s"]
        self._np = np
        self._ao = Mole.ao_loc_nr

    @property
    def nbas(self):
        return len(self._bas)

    def ao_loc_nr(self, cart=None):
        from ccsd_gpu_b200.gto.mole import Mole
        return Mole.ao_loc_nr(self, cart)

    def cart2sph_coeff(self):
        return self._c2s


@pytest.fixture(scope="session")
def golden_mols():
    import numpy as np
    out = {}
    for f in sorted(os.listdir(GOLDEN)):
        if f.startswith("eri_") and f.endswith(".npz") and "quartets" not in f:
            d = dict(np.load(os.path.join(GOLDEN, f)))
            out[f[4:-4]] = (GoldenMol(d), d)
    return out
