"""CPU oracle for the redfox_b200 kernels -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import this package.  It is the checker: a C restatement of the reference's algorithms
(``rfx_oracle.c``) plus, where the reference tree was present at build time, the
reference's own thrust entry files compiled for the CPU (``_ref/libredfox_ref.so``).
"""
from .binding import *  # noqa: F401,F403
