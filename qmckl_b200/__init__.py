"""qmckl_b200: the QMCkl orbital-evaluation path (AO VGL, MO VGL) on NVIDIA B200.

The product is the C-ABI library ``_lib/libqmckl_b200.so`` (headers in
``include/``).  ``qmckl_b200.qmckl`` is its Python face with the reference's
Python module conventions; ``qmckl_b200.gen`` builds the seeded benchmark
molecules; ``qmckl_b200.torch_ops`` exposes the adjoint to PyTorch autograd.
"""
__all__ = ["qmckl", "gen", "system"]
