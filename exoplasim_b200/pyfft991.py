"""Drop-in replacement for ExoPlaSim's f2py module ``exoplasim.pyfft991``.

pyburn imports this name instead of ``exoplasim.pyfft`` for NLAT 192 and 320
(pyburn.py:594-602).  The reference module differs from pyfft only in its
FFT (FFT991, pyfft991.f90:813-883); both compute the same real DFT with the
same packing and sqrt(2) scaling, and this library's one GPU FFT serves both,
so the functions are those of exoplasim_b200.pyfft.
"""
from .pyfft import (SQRT2, dv2uv, fc2gp, fc2sp, fc3gp, gp2fc, gp2sp, gp3fc, gpvsp, inigau, legini,  # noqa: F401
                    sp2fc, sp2fcdmu, sp2gp, sp3fc, spvgp, uv2dv)
