"""B200-native simulation core with the NeuronGPU API.

``neurongpu_b200.neurongpu`` is the drop-in Python interface (the reference's
``neurongpu`` module); ``neurongpu_b200.build`` compiles the CUDA library.
"""
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib",
                        "libneurongpu.so")

__all__ = ["LIB_PATH"]
