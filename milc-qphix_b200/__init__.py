"""qphix_b200: B200-native staggered (asqtad/HISQ) solver path behind the
QPhiX C API.  The product is the shared library ``lib/libqphix_b200.so``
(C ABI declared in ``include/``); this package holds its CUDA/C++ sources
(``csrc/``), the ctypes mirror of the C API used by tests and the benchmark
(``capi``) and the seeded synthetic inputs (``synthetic``)."""
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libqphix_b200.so")
