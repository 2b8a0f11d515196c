"""drape_b200: the quasi-static drape GPU stage (PTC + regularised Newton + block-Jacobi PCG + IPC contact) as
hand-written CUDA for NVIDIA B200 (sm_100a) behind a C ABI (include/drape_b200.h)."""
from .api import Drape, DrapeError, Options, default_options, load, version  # noqa: F401
