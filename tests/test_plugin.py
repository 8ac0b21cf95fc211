"""The GpuSpace engine plug-in (illuminaprt_b200/plugin/libilg_gpuspace.so)
on the CPU: it exports the reference's plug-in symbol set
(System/LibrarySymbols.h), the reference engine's PlugInManager registers it,
its "GPU" factory lands in the kernel's SpaceManager, and without a GPU the
space refuses to build (Build() false, with the CUDA reason) instead of
falling back to a CPU walk."""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from illuminaprt_b200 import build as pkg_build
from illuminaprt_b200 import scenes
from oracle import bindings

SYMBOLS = ["GetPlugInSingleton", "DisposePlugInSingleton", "CreatePlugInInstance", "GetPlugInInstance",
           "DisposePlugInInstance", "DisposePlugInInstances", "GpuSpaceLastError"]

needs_plugin = pytest.mark.skipif(not (os.path.exists(pkg_build.PLUGIN) and bindings.ref_available()),
                                  reason="plug-in or reference engine library not built")


def _cuda_present() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@needs_plugin
def test_plugin_exports_the_reference_symbol_set():
    # the plug-in leaves the engine's symbols to the host: load the engine first
    ctypes.CDLL(bindings.REF_SO, mode=ctypes.RTLD_GLOBAL)
    lib = ctypes.CDLL(pkg_build.PLUGIN)
    for name in SYMBOLS:
        assert hasattr(lib, name), name


@needs_plugin
def test_unknown_factory_is_reported():
    ref = bindings.RefLib()
    o = np.zeros((1, 4), np.float32)
    d = np.array([[0, 0, 1, 1e30]], np.float32)
    with pytest.raises(RuntimeError, match="no space factory named Nope"):
        ref.compare_spaces(pkg_build.PLUGIN, scenes.box_scene(), o, d, factory="Nope")


@needs_plugin
@pytest.mark.skipif(_cuda_present(), reason="checks the no-GPU failure path")
def test_gpu_space_fails_loudly_without_a_gpu():
    ref = bindings.RefLib()
    o = np.zeros((1, 4), np.float32)
    d = np.array([[0, 0, 1, 1e30]], np.float32)
    with pytest.raises(RuntimeError, match="Build returned false: GpuSpace: ilg_create"):
        ref.compare_spaces(pkg_build.PLUGIN, scenes.box_scene(), o, d)
