# Version of the gsplat2d Python API this package reproduces
# (gsplat2d/gsplat2d/version.py:1 in the reference).
__version__ = "0.1.11"
