"""B200-native AR4JA LDPC Monte Carlo engine (drop-in for the reference's scalar engine).

Modules: ``ar4ja`` (code construction), ``chinn`` (matrix files), ``capi`` (ctypes binding of the CUDA
library), ``sim`` (the ``ldpc_sim`` command line: getopt flags and JSON-lines protocol of the
reference engine), ``stats`` (confidence intervals), ``build`` (nvcc build of the library).
"""
__version__ = "0.1.0"
