"""Simulation parameters (src/utils/config.py of the reference).

The module-level names are the reference's (the drop-in reads them as
attributes of whatever `config` object it is given); the extra names select
the B200 step's options and default to the reference's behaviour.
"""
import types

# --- SIMULATION PARAMETERS (src/utils/config.py:9-14) ---
N_GRID = 128
N_BODIES = N_GRID ** 3
BOX_SIZE = 1.0
SOFTENING = 0.001
N_STEPS = 2500
A_START, A_END = 0.02, 1.0

# --- RENDER SETTINGS (src/utils/config.py:16-21) ---
ROTATION_SPEED = 0.001
CAM_DIST_MULT = 1.8
FOV = 60.0
RES = 1024
OUTPUT_DIR = "render_output"

# --- CUDA CONFIG (src/utils/config.py:23-27); validated, the library picks its own launch shapes ---
TPB = 256
BPG = (N_BODIES + TPB - 1) // TPB
BATCH_SIZE = int(5_000)
CACHE_SIZE = 256

# --- PHYSICS CONSTANTS (src/utils/config.py:29-34) ---
THETA = 0.7
G = 1.0
OMEGA_M = 1.0
OMEGA_L = 0.692
H0 = 67.8
STACK_SIZE_CHILD = 128

# --- B200 step options (no reference counterpart) ---
KEY_MODE = "compat30"      # "compat30": reference keys, bit-exact; "morton63": full 21-bit interleave
SORT_MODE = "auto"         # "full": radix sort every step; "adaptive": near-sorted path first (same
                           # argsort); "auto": adaptive for morton63 keys, full for compat30 keys
FORCE_MODE = "reference"   # "reference": per-particle stack traversal; "grouped": warp-per-bucket traversal
MAC = "ref_x"              # "ref_x": reference opening test; "periodic": 3-D extent + image-safe opening;
                           # "ewald": periodic (Ewald) force law instead of the minimum image, 3-D extent
PRECISION = "f32"          # per-particle traversal arithmetic: "f32" or "f64" (the reference's)
UPWARD = "plain"           # "plain": bit-exact upward pass; "compensated": two-sum + float64 root
BODIES_PER_LANE = 1        # grouped traversal: bodies per lane (buckets of 32 x this)
BLOCK_WARPS = 8            # grouped traversal: warps per block (2, 4 or 8)
QUADRUPOLE = False         # "ewald" test: internal nodes also apply their quadrupole moments
SUPER_BODIES = 0           # grouped "ref_x" traversal: super-bucket size of the two-level walk (0 = off)
SLAB_BODIES = 0            # periodic test: image-ambiguous nodes up to this many bodies' mass are
                           # applied with the per-pair minimum image (0 = exact)
SEED = 0                   # initial-condition seed
RES_W = None               # render width (None: RES)
RES_H = None               # render height (None: RES)


def make(**overrides):
    """A config namespace with this module's values and `overrides`.
    N_BODIES and BPG follow N_GRID unless given."""
    base = {k: v for k, v in globals().items() if k.isupper()}
    base.update(overrides)
    if "N_BODIES" not in overrides:
        base["N_BODIES"] = base["N_GRID"] ** 3
    if "BPG" not in overrides:
        base["BPG"] = (base["N_BODIES"] + base["TPB"] - 1) // base["TPB"]
    return types.SimpleNamespace(**base)
