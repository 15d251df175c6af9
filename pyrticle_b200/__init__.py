"""pyrticle_b200: the particle side of a pyrticle PIC step on NVIDIA B200.

Charge/current deposition (shape-function, normalised shape-function, brick
grid + remap), monomial field interpolation with the relativistic Lorentz
force and low-storage RK push, and particle-to-element location, behind the
reference's PicMethod / depositor / pusher API. Compute runs in libprt.so
(CUDA, sm_100a) through a C ABI (include/prt.h).
"""

__version__ = "0.1.0"
