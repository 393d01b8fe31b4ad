import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcytnx_b200.so")


def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def golden_bonds(z, mod):
    """Bonds of a golden fixture as `mod.Bond` objects (oracle or product)."""
    r = int(z["rank"])
    out = []
    for i in range(r):
        syms = [tuple(int(x) for x in s) for s in z[f"bond{i}_syms"]]
        if mod.__name__ == "oracle":
            out.append(mod.Bond(int(z[f"bond{i}_type"]), z[f"bond{i}_qnums"], z[f"bond{i}_degs"], syms))
        else:
            out.append(mod.Bond(int(z[f"bond{i}_type"]), z[f"bond{i}_qnums"], z[f"bond{i}_degs"],
                                [mod.Symmetry(s[0], s[1]) for s in syms]))
    return out


def golden_blocks(z):
    shapes = z["block_shapes"]
    data = z["data"]
    blocks, pos = [], 0
    for s in shapes:
        n = int(np.prod(s))
        blocks.append(data[pos:pos + n].reshape(s))
        pos += n
    return blocks


def golden_oracle_tensor(name, labels=None):
    import oracle as O

    z = load_golden(name)
    t = O.BlockTensor(golden_bonds(z, O), list(z["labels"]), int(z["rowrank"]), z["itoi"], golden_blocks(z))
    return t.relabel(labels) if labels else t
