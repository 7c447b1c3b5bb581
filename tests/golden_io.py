"""Loads the committed golden vectors (tests/golden/*.npz)."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def job_sets():
    return sorted(os.path.basename(p)[5:-4] for p in glob.glob(os.path.join(GOLDEN, "jobs_*.npz")))


def seed_sets():
    return sorted(os.path.basename(p)[6:-4] for p in glob.glob(os.path.join(GOLDEN, "seeds_*.npz")))


def load_jobs(name):
    z = np.load(os.path.join(GOLDEN, f"jobs_{name}.npz"))
    return z["u8"], z["jobs"], z["score"], z["ext"]


def load_seeds(name):
    z = np.load(os.path.join(GOLDEN, f"seeds_{name}.npz"))
    return z["u8"], z["seeds"], z["opt"], z["reg"]


def sw_sets():
    return sorted(os.path.basename(p)[3:-4] for p in glob.glob(os.path.join(GOLDEN, "sw_*.npz")))


def load_sw(name):
    z = np.load(os.path.join(GOLDEN, f"sw_{name}.npz"))
    return z["u8"], z["jobs"], z["score"], z["xtras"], z["out"]


def load_rows(kind, name):
    """The golden file of a row around the extension (chains_, global_, tbpairs_, seedflt_) as a
    dict of arrays."""
    z = np.load(os.path.join(GOLDEN, f"{kind}_{name}.npz"))
    return {k: z[k] for k in z.files}


def row_sets(kind):
    return sorted(os.path.basename(p)[len(kind) + 1:-4] for p in glob.glob(os.path.join(GOLDEN, f"{kind}_*.npz")))


def workload(d):
    """The ChainWorkload stored in a golden file."""
    from g3sa_b200.chains import ChainWorkload
    return ChainWorkload(d["u8"], int(d["l_pac"]), d["anns"], d["reads"], d["chains"], d["seeds"])
