"""B200 Lagrangian parcel step (SCALE-TRACK hot path): package directory.

The product is libscaletrack.so (csrc/, C ABI in include/scaletrack.h); scaletrack.py is
its Python host side.  Importing this package loads nothing on its own.
"""
