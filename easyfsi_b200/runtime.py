"""Process-wide runtime of the B200 path (replaces simulation_core/runtime.py).

``TaichiRuntimeConfig`` keeps the reference's name and fields so callers that
build one keep working; here it selects the CUDA device instead of a Taichi
backend.  Like the reference (runtime.py:24-59) the first initialisation wins,
the CPU backend is refused and a different ``default_fp`` later is an error.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _native

_SUPPORTED_ARCHS = ("cuda", "gpu")
_SUPPORTED_FPS = ("f32", "f64")

# dtype tokens (the reference compares field dtypes against ti.f32 / ti.f64 / ti.i32)
f32 = torch.float32
f64 = torch.float64
i32 = torch.int32


@dataclass(frozen=True)
class TaichiRuntimeConfig:
    arch: str = "cuda"
    default_fp: str = "f32"
    random_seed: int = 0


RuntimeConfig = TaichiRuntimeConfig

_STATE = {"initialized": False, "fp": None, "device": None}


def init_runtime(config: TaichiRuntimeConfig | None = None) -> torch.device:
    """Initialise once; return the CUDA device all fields live on."""
    cfg = config or TaichiRuntimeConfig()
    arch = str(cfg.arch).lower()
    if arch == "cpu":
        raise ValueError("easyfsi_b200 is GPU-only; use arch='cuda' or arch='gpu'")
    if arch not in _SUPPORTED_ARCHS:
        raise ValueError(f"unsupported arch: {cfg.arch!r}")
    fp = str(cfg.default_fp)
    if fp not in _SUPPORTED_FPS:
        raise ValueError(f"unsupported default_fp: {cfg.default_fp!r}; expected one of {_SUPPORTED_FPS}")
    if _STATE["initialized"]:
        if _STATE["fp"] != fp:
            raise ValueError(
                f"runtime is already initialized with default_fp={_STATE['fp']!r}; "
                f"cannot re-initialize with default_fp={fp!r}"
            )
        return _STATE["device"]
    if not torch.cuda.is_available():
        raise RuntimeError("easyfsi_b200 requires a CUDA device (B200, sm_100a); none is visible")
    _native.load()
    torch.manual_seed(int(cfg.random_seed))
    device = torch.device("cuda", torch.cuda.current_device())
    _STATE.update(initialized=True, fp=fp, device=device)
    return device


# The reference's entry point name.
init_taichi = init_runtime


def current_stream_handle() -> int:
    return torch.cuda.current_stream().cuda_stream


class StepGraph:
    """A whole coupled step as one CUDA graph (``efsi_step_graph_*``; no
    reference counterpart).  ``capture(step)`` runs ``step`` once under a
    stream capture on a stream of its own -- every library launch of the step
    is recorded, PCG solves run their device-side loop -- and ``launch()``
    replays it on the current stream.  The step must make no host reads and
    allocate nothing: run it once eagerly first, and keep its reports off."""

    def __init__(self) -> None:
        self._handle = None
        self._stream = None

    def capture(self, step) -> None:
        from ctypes import byref, c_void_p

        self.close()
        self._stream = torch.cuda.Stream()
        self._stream.wait_stream(torch.cuda.current_stream())
        handle = c_void_p()
        with torch.cuda.stream(self._stream):
            _native.call("efsi_step_graph_begin", c_void_p(self._stream.cuda_stream))
            try:
                step()
            finally:
                _native.call("efsi_step_graph_end", c_void_p(self._stream.cuda_stream), byref(handle))
        self._handle = handle

    def launch(self) -> None:
        from ctypes import c_void_p

        if self._handle is None:
            raise RuntimeError("no step graph has been captured")
        _native.call("efsi_step_graph_launch", self._handle, c_void_p(torch.cuda.current_stream().cuda_stream))

    def close(self) -> None:
        if self._handle is not None and self._handle.value:
            _native.call("efsi_step_graph_destroy", self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchStepGraph:
    """Independent coupled steps (one per instance) as ONE CUDA graph: the
    capture forks a stream per instance from its origin stream and joins them
    all back, so the graph holds one independent branch per instance and a
    single launch advances every instance; branches of uneven size run
    concurrently on the GPU.  Each instance's pressure solve must run its
    device-side loop (``device_loop_solves``), and each step must make no
    host reads and allocate nothing (run every step once eagerly first and
    keep the reports off).  No reference counterpart."""

    def __init__(self) -> None:
        self._handle = None
        self._streams = []

    def capture(self, steps) -> None:
        from ctypes import byref, c_void_p

        self.close()
        origin = torch.cuda.Stream()
        origin.wait_stream(torch.cuda.current_stream())
        streams = [torch.cuda.Stream() for _ in steps]
        handle = c_void_p()
        with torch.cuda.stream(origin):
            _native.call("efsi_step_graph_begin", c_void_p(origin.cuda_stream))
            try:
                fork = torch.cuda.Event()
                fork.record(origin)
                joins = []
                for st, step in zip(streams, steps):
                    st.wait_event(fork)
                    with torch.cuda.stream(st):
                        step()
                    ev = torch.cuda.Event()
                    ev.record(st)
                    joins.append(ev)
                for ev in joins:
                    origin.wait_event(ev)
            finally:
                _native.call("efsi_step_graph_end", c_void_p(origin.cuda_stream), byref(handle))
        self._handle = handle
        self._streams = [origin] + streams

    def launch(self) -> None:
        from ctypes import c_void_p

        if self._handle is None:
            raise RuntimeError("no batch step graph has been captured")
        _native.call("efsi_step_graph_launch", self._handle, c_void_p(torch.cuda.current_stream().cuda_stream))

    def close(self) -> None:
        if self._handle is not None and self._handle.value:
            _native.call("efsi_step_graph_destroy", self._handle)
        self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
