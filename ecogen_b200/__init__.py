"""ecogen_b200: the explicit finite-volume step of ECOGEN (Cartesian meshes) on NVIDIA B200.

The product is the CUDA library ``libecg.so`` with the C ABI of ``include/ecogen_b200.h``;
``api`` binds it from Python and ``cases`` writes ECOGEN-format case inputs.
"""
__all__ = ["api", "cases"]
