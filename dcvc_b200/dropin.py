"""Registers this package's drop-in modules under the reference's module names.

    import dcvc_b200.dropin
    dcvc_b200.dropin.install()
    # from here on, `import inference_extensions_cuda` / `import MLCodec_extensions_cpp` in the
    # reference's models (src/models/video_model_ht.py:419-427, entropy_models.py:34,40) resolve
    # to dcvc_b200's implementations.
"""
import sys

from . import MLCodec_extensions_cpp, inference_extensions_cuda

NAMES = {"inference_extensions_cuda": inference_extensions_cuda,
         "MLCodec_extensions_cpp": MLCodec_extensions_cpp}


def install():
    for name, mod in NAMES.items():
        sys.modules[name] = mod


def uninstall():
    for name, mod in NAMES.items():
        if sys.modules.get(name) is mod:
            del sys.modules[name]
