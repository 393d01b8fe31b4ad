"""Convert the reference's binary test fixtures for the hot path into small .npz files.

Run where a checkout of the reference exists, giving its root as the argument (or in
the environment variable CYTNX_REFERENCE_ROOT); the GPU-side tests only read the .npz
files written here.

Fixtures converted (the reference tests that use them):

* BlockUniTensor contract_{L,R,ans}{1,2,3}  -- tests/BlockUniTensor_test.cpp:679-717
* BlockUniTensor permute_T{1,2,3} / permute_ans{1,2,3} -- tests/BlockUniTensor_test.cpp:308-360
* DenseUniTensor denseutensor{1,2}, densecontres{1,2,3}, densepermu{1,2}
                                               -- tests/DenseUniTensor_test.cpp:2594-2619
* linalg/Lanczos_Gnd lan_block_{A,B,C}         -- tests/linalg_test/Lanczos_Gnd_test.cpp:102-125,392-445
* linalg/Svd_truncate Svd_truncate1 + S_truncate1 -- tests/linalg_test/linalg_test.h:78-83, linalg_test.cpp:57-67
* common/sym_UT_U1_exp_Svals_F64 with its linalg/Svd_truncate answers (singular values, reconstructed
  tensor, and the min_blockdim variants)       -- tests/linalg_test/Gesvd_truncate_test.cpp:107-135, 187-270

Usage:  python tests/golden/make_golden.py [reference_root]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from cytnx_b200 import fileio  # noqa: E402


def pack_unitensor(u):
    out = {
        "uten_type": np.int64(u["uten_type"]),
        "rowrank": np.int64(u["rowrank"]),
        "is_diag": np.bool_(u["is_diag"]),
        "labels": np.array(u["labels"], dtype="U"),
        "rank": np.int64(len(u["labels"])),
    }
    for i, b in enumerate(u["bonds"]):
        out[f"bond{i}_type"] = np.int64(b["type"])
        out[f"bond{i}_qnums"] = np.asarray(b["qnums"], dtype=np.int64)
        out[f"bond{i}_degs"] = np.asarray(b["degs"], dtype=np.int64)
        out[f"bond{i}_syms"] = np.array([[s["stype"], s["n"]] for s in b["syms"]], dtype=np.int64).reshape(-1, 2)
        out[f"bond{i}_dim"] = np.int64(b["dim"])
    if u["uten_type"] == fileio.UTEN_BLOCK:
        blocks = u["blocks"]
        out["itoi"] = np.asarray(u["itoi"], dtype=np.int64)
        out["block_shapes"] = np.array([b.shape for b in blocks], dtype=np.int64).reshape(len(blocks), -1)
        out["data"] = np.concatenate([b.ravel() for b in blocks]) if blocks else np.zeros(0)
    else:
        out["block"] = u["block"]
    return out


def main(ref_root: str) -> None:
    base = os.path.join(ref_root, "tests", "test_data_base")
    jobs = []
    bdir = os.path.join(base, "common", "BlockUniTensor")
    for stem in ["contract_L1", "contract_R1", "contract_ans1", "contract_L2", "contract_R2",
                 "contract_ans2", "contract_L3", "contract_R3", "contract_ans3",
                 "permute_T1", "permute_ans1", "permute_T2", "permute_ans2",
                 "permute_T3", "permute_ans3"]:
        jobs.append((os.path.join(bdir, stem + ".cytnx"), "block_" + stem))
    ddir = os.path.join(base, "common", "DenseUniTensor")
    for stem in ["denseutensor1", "denseutensor2", "densecontres1", "densecontres2",
                 "densecontres3", "densepermu1", "densepermu2"]:
        jobs.append((os.path.join(ddir, stem + ".cytnx"), "dense_" + stem))
    for src, dst in jobs:
        u = fileio.read_unitensor(src)
        np.savez_compressed(os.path.join(HERE, dst + ".npz"), **pack_unitensor(u))
        print("wrote", dst)
    sdir = os.path.join(base, "linalg", "Svd_truncate")
    jobs_svd = [(os.path.join(sdir, "Svd_truncate1.cytnx"), "svd_truncate1_T"),
                (os.path.join(base, "common", "sym_UT_U1_exp_Svals_F64.cytnx"), "svd_u1_exp_src")]
    for suffix in ["", "_reconstructed", "_minblockdim", "_minblockdim_reconstructed"]:
        jobs_svd.append((os.path.join(sdir, f"sym_UT_U1_exp_Svals_F64{suffix}.cytnx"), f"svd_u1_exp_ans{suffix}"))
    for src, dst in jobs_svd:
        u = fileio.read_unitensor(src)
        np.savez_compressed(os.path.join(HERE, dst + ".npz"), **pack_unitensor(u))
        print("wrote", dst)
    np.savez_compressed(os.path.join(HERE, "svd_truncate1_S.npz"),
                        S=fileio.read_tensor(os.path.join(sdir, "S_truncate1.cytn")))
    print("wrote svd_truncate1_S")
    ldir = os.path.join(base, "linalg", "Lanczos_Gnd")
    lan = {k: fileio.read_tensor(os.path.join(ldir, f"lan_block_{k}.cytn")) for k in "ABC"}
    np.savez_compressed(os.path.join(HERE, "lanczos_blocks.npz"), **lan)
    print("wrote lanczos_blocks")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CYTNX_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: python tests/golden/make_golden.py <reference_root> (or set CYTNX_REFERENCE_ROOT)")
    main(root)
