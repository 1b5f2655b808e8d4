"""Mirror of syclfft's plan API over the B200 provider's C ABI.

Reference surface and semantics followed here:
  include/syclfft/common.hpp:34-93    enums (values kept), plan_options, error_code
  include/syclfft/syclfft.hpp:45-130  plan<Scalar>, plan_many_dft / plan_dft_1d/2d/3d
  src/sycl/sycl.cpp:424-491           plan construction, direction check, provider selection
  src/sycl/sycl.cpp:615-641           execute: pointer validation, placement rules,
                                      per-plan serialisation on the previous execution
  src/sycl/sycl.cpp:818-874           execute overloads, moved-from plan -> invalid_state
  src/sycl/sycl.cpp:901-907           scratch_size_bytes
  src/core/provider_loader.cpp:112-132 checked_element_count errors
"""
from __future__ import annotations

import ctypes
import enum
import json
import sys
import threading
import weakref
from dataclasses import dataclass

from . import _provider

try:  # CPython fast call into the provider's execute entry (csrc/fastcall.c); ctypes otherwise
    from . import _fastcall
except ImportError:  # pragma: no cover - the Makefile builds it beside this file
    _fastcall = None


class direction(enum.IntEnum):
    forward = -1
    backward = 1


class placement(enum.IntEnum):
    in_place = 0
    out_of_place = 1


class normalization(enum.IntEnum):
    none = 0
    forward = 1
    backward = 2
    orthogonal = 3


class planning_mode(enum.IntEnum):
    estimate = 0
    measure = 1


class provider(enum.IntEnum):
    automatic = 0
    portable_sycl = 1
    fftw = 2
    cufft = 3
    rocfft = 4
    onemkl = 5
    b200 = 6


class error_code(enum.IntEnum):
    invalid_argument = 0
    invalid_state = 1
    invalid_pointer = 2
    unsupported_precision = 3
    provider_unavailable = 4
    planning_failed = 5
    execution_failed = 6
    plugin_error = 7


class SyclfftError(RuntimeError):
    """syclfft::exception: a message plus an error_code."""

    def __init__(self, code: error_code, message: str):
        super().__init__(message)
        self.code = error_code(code)


@dataclass
class plan_options:
    placement: placement = placement.out_of_place
    normalization: normalization = normalization.none
    planning: planning_mode = planning_mode.estimate
    preferred_provider: provider = provider.automatic
    # B200 extension (no counterpart in syclfft::plan_options): complex<float> plans run the
    # radix-16 butterflies of eligible axes (256 / 4096 points) as BF16 hi/lo matrix products
    # with FP32 accumulation on the tensor cores; ignored for complex<double>.
    split_precision: bool = False


@dataclass
class data_layout:
    """B200 extension (the reference's plans read and write contiguous batch-major arrays only):
    element (b, i0, .., i_{rank-1}) of the input sits at b * in_distance + sum_k i_k * in_strides[k]
    complex elements from the input's start, and likewise for the output. FFTW's advanced
    interface (istride/idist, ostride/odist) generalised to one stride per axis."""
    in_strides: tuple
    in_distance: int
    out_strides: tuple
    out_distance: int

    @staticmethod
    def contiguous(lengths):
        strides, step = [], 1
        for n in reversed([int(v) for v in lengths]):
            strides.insert(0, step)
            step *= n
        return data_layout(tuple(strides), step, tuple(strides), step)

    def _side(self, output):
        return (tuple(int(v) for v in (self.out_strides if output else self.in_strides)),
                int(self.out_distance if output else self.in_distance))

    def extent(self, lengths, batch, output):
        """Elements a buffer must hold for this side: 1 + the largest offset."""
        strides, dist = self._side(output)
        return 1 + sum((int(n) - 1) * s for n, s in zip(lengths, strides)) + (int(batch) - 1) * dist

    def check(self, lengths, batch, in_place):
        for output in (False, True):
            strides, dist = self._side(output)
            side = "output" if output else "input"
            if len(strides) != len(lengths):
                raise SyclfftError(error_code.invalid_argument, f"{side} layout needs one stride per axis")
            if any(s < 1 for s in strides):
                raise SyclfftError(error_code.invalid_argument, f"{side} strides must be >= 1")
            if batch > 1 and dist < 1:
                raise SyclfftError(error_code.invalid_argument, f"{side} distance must be >= 1")
        # the output must not write two elements to one address: sorted by stride, each stride
        # has to exceed the span of the smaller ones
        strides, dist = self._side(True)
        dims = sorted([(s, int(n)) for s, n in zip(strides, lengths) if int(n) > 1] +
                      ([(dist, int(batch))] if batch > 1 else []))
        reach = 0
        for s, n in dims:
            if s <= reach:
                raise SyclfftError(error_code.invalid_argument, "output layout overlaps itself")
            reach += s * (n - 1)
        if in_place:
            same = all(a == b for a, b, n in zip(self.in_strides, self.out_strides, lengths) if int(n) > 1)
            if not same or (batch > 1 and self.in_distance != self.out_distance):
                raise SyclfftError(error_code.invalid_argument, "an in-place plan needs equal input and output layouts")


def _torch():
    import torch
    return torch


_EVENT_CLS = None
_EVENT_BASE_RECORD = None


def _event_class():
    """ExecutionEvent: the torch.cuda.Event an execute returns (the stand-in for sycl::event),
    which also reports a failed device wait. A bounded wait in a plan's kernel that gave up
    leaves that execution's output incomplete and sets the plan's status word; the reference
    reports a failed provider execution as error_code::execution_failed (src/sycl/sycl.cpp:
    671-676), and so do synchronize() and wait_and_throw() here, once per failure."""
    global _EVENT_CLS
    if _EVENT_CLS is None:
        torch = _torch()

        class ExecutionEvent(torch.cuda.Event):
            def __new__(cls, lib=None, plans=()):
                self = super().__new__(cls)
                self._lib = lib
                self._plans = plans  # kept alive while the event is: their status words are read
                return self

            def synchronize(self):
                super().synchronize()
                self._check()

            def wait_and_throw(self):
                self.synchronize()

            def _check(self):
                for p in self._plans:
                    h = getattr(p, "_handle", None)
                    if not h:
                        continue  # closed or moved from: nothing left to report
                    code = self._lib.syclfft_b200_plan_take_status(h)
                    if code > 0:
                        raise SyclfftError(error_code.execution_failed,
                                           f"a bounded wait in a B200 kernel gave up (status {code}); the output of "
                                           "this execution is incomplete")

        _EVENT_CLS = ExecutionEvent
        global _EVENT_BASE_RECORD
        _EVENT_BASE_RECORD = torch._C._CudaEventBase.record  # record(event, stream), no current-stream lookup
    return _EVENT_CLS


_STREAMS = {}  # (device, raw cudaStream_t) -> torch.cuda.Stream: events are recorded through these


def _stream_object(torch, handle, device, given=None):
    """A torch.cuda.Stream for the raw stream `handle` of `device` (cached: building one from
    the current-stream query costs more than the rest of a small execute)."""
    key = (device, handle)
    s = _STREAMS.get(key)
    if s is None:
        s = given
        if s is None:
            cur = torch.cuda.current_stream(device)
            s = cur if cur.cuda_stream == handle else torch.cuda.ExternalStream(handle, device=device)
        if len(_STREAMS) > 256:
            _STREAMS.clear()
        _STREAMS[key] = s
    return s


def _host_tensor(t):
    """True for a page-locked (pinned) CPU tensor: host USM in the reference's terms."""
    torch = _torch()
    return isinstance(t, torch.Tensor) and not t.is_cuda


def execute_host(stages, input, output=None, batch=None, stream=None):
    """Run `stages` -- (plan, direction or None, normalization or None) tuples, or plans -- one
    after the other on transforms held in page-locked host tensors (B200 extension over the
    reference's host-USM execute, sycl.cpp:72-85). The batch streams through the device in
    chunks: copy in, the stages, copy out, on overlapping streams. `output` defaults to
    `input` (in place). Returns the completion event (an ExecutionEvent)."""
    torch = _torch()
    items = []
    for st in stages:
        plan, d, n = (st, None, None) if isinstance(st, Plan) else (tuple(st) + (None, None))[:3]
        if not getattr(plan, "_handle", None):
            raise SyclfftError(error_code.invalid_state, "Cannot execute a moved-from plan")
        items.append((plan, 0 if d is None else int(d), -1 if n is None else int(n)))
    if not items:
        raise SyclfftError(error_code.invalid_argument, "at least one stage is needed")
    first = items[0][0]
    output = input if output is None else output
    for t, name in ((input, "input"), (output, "output")):
        if not isinstance(t, torch.Tensor) or t.is_cuda:
            raise SyclfftError(error_code.invalid_pointer, f"{name} must be a page-locked host tensor")
        if not t.is_pinned():
            raise SyclfftError(error_code.invalid_pointer,
                               f"{name} is pageable host memory; host buffers must be page-locked (pin_memory)")
        if t.dtype != first.dtype:
            raise SyclfftError(error_code.invalid_argument, f"{name} has dtype {t.dtype}, plan needs {first.dtype}")
    b = first._batch if batch is None else int(batch)
    need = b * (first._elements // first._batch)
    for t, name in ((input, "input"), (output, "output")):
        if not t.is_contiguous() or t.numel() < need:
            raise SyclfftError(error_code.invalid_argument, f"{name} must be contiguous with >= {need} elements")
    arr = (_provider.HostStageV1 * len(items))()
    for i, (plan, d, n) in enumerate(items):
        arr[i].plan, arr[i].direction, arr[i].normalization = plan._handle, d, n
    s = stream or torch.cuda.current_stream(first._device)
    locks = sorted({id(p): p for p, _, _ in items}.values(), key=id)
    for p in locks:
        p._lock.acquire()
    try:
        for p in locks:
            if p._last_event is not None:
                s.wait_event(p._last_event)
        err = ctypes.create_string_buffer(_provider.ERR_CAP)
        rc = first._lib.syclfft_b200_execute_host(arr, len(items), input.data_ptr(), output.data_ptr(), b,
                                                  s.cuda_stream, err, _provider.ERR_CAP)
        if rc != 0 or err.value:
            raise SyclfftError(error_code.execution_failed, err.value.decode() or "execution failed")
        ev = _event_class()(first._lib, tuple(locks))
        ev.record(s)
        for p in locks:
            p._last_event = ev
            p._last_stream = s.cuda_stream
        return ev
    finally:
        for p in locks:
            p._lock.release()


def _checked_element_count(lengths, batch):
    if len(lengths) == 0 or len(lengths) > 3:
        raise SyclfftError(error_code.invalid_argument, "FFT rank must be between 1 and 3")
    if batch == 0:
        raise SyclfftError(error_code.invalid_argument, "FFT batch count must be non-zero")
    count = int(batch)
    for n in lengths:
        if n == 0:
            raise SyclfftError(error_code.invalid_argument, "FFT dimensions must be non-zero")
        count *= int(n)
        if count >= 1 << 64:
            raise SyclfftError(error_code.invalid_argument, "FFT element count overflows size_t")
    return count


class Plan:
    """syclfft::plan<Scalar> over the B200 provider. `scalar` is "float" or "double"."""

    def __init__(self, scalar: str, lengths, batch_count: int, dir, options: plan_options | None = None,
                 device: int | None = None, layout: data_layout | None = None):
        options = options or plan_options()
        if scalar not in ("float", "double"):
            raise SyclfftError(error_code.unsupported_precision, "syclfft supports float and double precision")
        self._lengths = [int(v) for v in lengths]
        self._batch = int(batch_count)
        self._elements = _checked_element_count(self._lengths, self._batch)
        self._extent = {"input": self._elements, "output": self._elements}
        if layout is not None:
            layout.check(self._lengths, self._batch, options.placement == placement.in_place)
            self._extent = {"input": layout.extent(self._lengths, self._batch, False),
                            "output": layout.extent(self._lengths, self._batch, True)}
        try:
            self._direction = direction(int(dir))
        except ValueError:
            raise SyclfftError(error_code.invalid_argument, "Invalid FFT direction") from None
        self._options = options
        self._double = scalar == "double"
        if options.preferred_provider not in (provider.automatic, provider.b200):
            raise SyclfftError(error_code.provider_unavailable,
                               f"{provider(options.preferred_provider).name} provider is not part of this build")
        torch = _torch()
        if not torch.cuda.is_available():
            raise SyclfftError(error_code.provider_unavailable, "no CUDA device is available")
        self._device = torch.cuda.current_device() if device is None else int(device)
        try:
            self._lib = _provider.load()
        except OSError as e:
            raise SyclfftError(error_code.provider_unavailable, str(e)) from None
        self._api = _provider.provider(self._lib)
        if self._api.abi_version != _provider.ABI_VERSION:
            raise SyclfftError(error_code.plugin_error, "B200 provider ABI mismatch")
        err = ctypes.create_string_buffer(_provider.ERR_CAP)
        if not self._api.supports(self._device, err, _provider.ERR_CAP):
            raise SyclfftError(error_code.provider_unavailable, err.value.decode() or "device not supported")
        cfg = _provider.make_config(self._lengths, self._batch, int(self._direction), self._double,
                                    options.placement == placement.in_place, int(options.normalization),
                                    options.planning == planning_mode.measure, self._device)
        self._cfg = cfg
        flags = _provider.CREATE_SYNC | (_provider.CREATE_SPLIT_BF16 if options.split_precision else 0)
        if layout is not None:
            lay = _provider.LayoutV1()
            for k, v in enumerate(layout.in_strides):
                lay.in_strides[k] = int(v)
            for k, v in enumerate(layout.out_strides):
                lay.out_strides[k] = int(v)
            lay.in_distance, lay.out_distance = int(layout.in_distance), int(layout.out_distance)
            h = self._lib.syclfft_b200_create_strided(ctypes.byref(cfg), ctypes.byref(lay), flags, err,
                                                      _provider.ERR_CAP)
        elif options.split_precision and not self._double:
            h = self._lib.syclfft_b200_create_ex(ctypes.byref(cfg), flags, err, _provider.ERR_CAP)
        else:
            h = self._api.create(ctypes.byref(cfg), err, _provider.ERR_CAP)
        if not h:
            raise SyclfftError(error_code.planning_failed, err.value.decode() or "B200 plan creation failed")
        self._handle = h
        self._lock = threading.Lock()
        self._last_event = None
        self._last_stream = None
        self._err = ctypes.create_string_buffer(_provider.ERR_CAP)
        self._execute = self._api.execute
        self._bind_fast_path()

    def _bind_fast_path(self):
        self._checked = {}  # name -> (weak tensor, data_ptr, numel) of the last validated buffer
        self._events = []   # ExecutionEvents this plan may record again once nobody holds them
        self._exec_addr = ctypes.cast(self._execute, ctypes.c_void_p).value
        self._err_addr = ctypes.addressof(self._err)

    def _event(self, capturing):
        """An ExecutionEvent to record: one of this plan's earlier events that nothing outside
        the plan references any more (re-recording it is then unobservable), else a new one."""
        if not capturing:
            for e in self._events:
                if sys.getrefcount(e) <= 3:  # the list, the loop variable and the argument
                    return e
        ev = (_EVENT_CLS or _event_class())(self._lib, (self,))
        if not capturing and len(self._events) < 4:
            self._events.append(ev)
        return ev

    # -- properties (syclfft.hpp:62-66) --
    def shape(self):
        return list(self._lengths) if self._handle else []

    def batch_count(self):
        return self._batch if self._handle else 0

    def direction(self):
        return self._direction if self._handle else direction.forward

    def selected_provider(self):
        return provider.b200 if self._handle else provider.automatic

    def scratch_size_bytes(self):
        return int(self._api.scratch_bytes(self._handle)) if self._handle else 0

    @property
    def elements(self):
        return self._elements

    @property
    def dtype(self):
        return _torch().complex128 if self._double else _torch().complex64

    def describe(self) -> dict:
        buf = ctypes.create_string_buffer(1 << 16)
        n = self._lib.syclfft_b200_describe_plan(self._handle, buf, 1 << 16)
        if n < 0:
            raise SyclfftError(error_code.invalid_state, "plan description unavailable")
        return json.loads(buf.value.decode())

    def launches(self) -> int:
        return int(self._lib.syclfft_b200_plan_launches(self._handle))

    # -- execution (sycl.cpp:615-641, 818-874) --
    def _pointer(self, t, name):
        # the buffer validated last time, unchanged: same tensor object, storage and size
        c = self._checked.get(name)
        if c is not None and c[0]() is t:
            ptr = t.data_ptr()
            if ptr == c[1] and t.numel() == c[2] and t.is_contiguous():
                return ptr
        ptr = self._validate_pointer(t, name)
        if not isinstance(t, int):
            self._checked[name] = (weakref.ref(t), ptr, t.numel())
        return ptr

    def _validate_pointer(self, t, name):
        torch = _torch()
        if t is None:
            raise SyclfftError(error_code.invalid_pointer, f"{name} must be non-null")
        if isinstance(t, int):
            if t == 0:
                raise SyclfftError(error_code.invalid_pointer, f"{name} must be non-null")
            return t
        if not isinstance(t, torch.Tensor):
            raise SyclfftError(error_code.invalid_pointer, f"{name} is not a device allocation in the plan context")
        if t.is_cuda:
            if t.get_device() != self._device:
                raise SyclfftError(error_code.invalid_pointer, f"{name} lives on another device than the plan")
        elif not t.is_pinned():  # page-locked host memory is device-accessible (read over the bus)
            raise SyclfftError(error_code.invalid_pointer, f"{name} is not a device allocation in the plan context")
        dtype = torch.complex128 if self._double else torch.complex64
        if t.dtype != dtype:
            raise SyclfftError(error_code.invalid_argument, f"{name} has dtype {t.dtype}, plan needs {dtype}")
        need = self._extent[name]
        if not t.is_contiguous() or t.numel() < need:
            raise SyclfftError(error_code.invalid_argument, f"{name} must be contiguous with >= {need} elements")
        return t.data_ptr()

    def execute(self, a, b=None, dependencies=None, stream=None):
        """execute(inout[, deps]) for in-place plans, execute(input, output[, deps]) otherwise.

        Buffers are CUDA tensors or raw device pointers; page-locked host tensors on both sides
        (host USM, which the reference's execute accepts, sycl.cpp:72-85) stream through the
        device in overlapped chunks (execute_host); a page-locked host tensor on one side only
        is read or written by the kernels directly over the bus. Returns an ExecutionEvent."""
        if not getattr(self, "_handle", None):
            raise SyclfftError(error_code.invalid_state, "Cannot execute a moved-from plan")
        # pointers are validated before the placement rules, as sycl.cpp:619-635 does
        if a is None or (isinstance(a, int) and a == 0):
            raise SyclfftError(error_code.invalid_pointer, "input must be non-null")
        if isinstance(b, int) and b == 0:
            raise SyclfftError(error_code.invalid_pointer, "output must be non-null")
        one_pointer = b is None
        pl = self._options.placement
        if pl == placement.in_place and not one_pointer:
            raise SyclfftError(error_code.invalid_argument, "In-place plan must be executed with execute(inout)")
        if pl == placement.out_of_place and one_pointer:
            raise SyclfftError(error_code.invalid_argument, "Out-of-place plan requires input and output arguments")
        if _host_tensor(a) and (one_pointer or _host_tensor(b)) and not isinstance(self, RealPlan) \
                and self._extent["input"] == self._elements and self._extent["output"] == self._elements:
            if pl == placement.out_of_place and a.data_ptr() == b.data_ptr():
                raise SyclfftError(error_code.invalid_argument, "Out-of-place plan requires distinct allocations")
            torch = _torch()
            s = stream or torch.cuda.current_stream(self._device)
            for dep in dependencies or ():
                s.wait_event(dep)
            return execute_host([self], a, a if one_pointer else b, stream=s)
        inp = self._pointer(a, "input")
        out = inp if one_pointer else self._pointer(b, "output")
        if pl == placement.out_of_place and inp == out:
            raise SyclfftError(error_code.invalid_argument, "Out-of-place plan requires distinct allocations")
        torch = _torch()
        dev = self._device
        tc = torch._C
        if stream is None and tc._cuda_getDevice() == dev:
            # the current stream of the current device: its raw handle and capture state
            # without building a Stream object
            s = None
            handle = tc._cuda_getCurrentRawStream(dev)
            capturing = tc._cuda_isCurrentStreamCapturing()
        else:
            current = torch.cuda.current_stream(dev)
            s = stream or current
            handle = s.cuda_stream
            if s is current or s == current:
                with torch.cuda.device(dev):
                    capturing = torch.cuda.is_current_stream_capturing()
            else:
                with torch.cuda.stream(s):
                    capturing = torch.cuda.is_current_stream_capturing()
        with self._lock:
            for dep in dependencies or ():
                s = s or _stream_object(torch, handle, dev)
                s.wait_event(dep)
            if self._last_event is not None and not capturing and self._last_stream != handle:
                # A graph cannot depend on work outside its capture; captured launches run
                # only at replay, which the caller orders against earlier executes. On the
                # stream of the previous execute, stream order already serialises them.
                s = s or _stream_object(torch, handle, dev)
                s.wait_event(self._last_event)
            err = self._err
            # the provider writes the error buffer only on failure (a non-zero return)
            if _fastcall is not None:
                rc = _fastcall.execute(self._exec_addr, self._handle, inp, out, handle, self._err_addr,
                                       _provider.ERR_CAP)
            else:
                rc = self._execute(self._handle, inp, out, handle, err, _provider.ERR_CAP)
            if rc != 0:
                raise SyclfftError(error_code.execution_failed, err.value.decode() or "execution failed")
            ev = self._event(capturing)
            _EVENT_BASE_RECORD(ev, _stream_object(torch, handle, dev, s))
            # an event recorded inside a capture belongs to the graph: ordering of replays
            # against later executes is the caller's, as for any captured work
            self._last_event = None if capturing else ev
            self._last_stream = None if capturing else handle
            return ev

    def close(self):
        h = getattr(self, "_handle", None)
        if h:
            if self._last_event is not None:
                try:
                    self._last_event.synchronize()
                except SyclfftError:
                    pass  # a failed wait was already reported or is moot once the plan goes
            self._api.destroy(h)
            self._handle = None

    def move(self) -> "Plan":
        """C++ move: returns a new owner, leaves this plan moved-from (invalid_state on execute)."""
        other = object.__new__(Plan)
        other.__dict__.update(self.__dict__)
        self._handle = None
        return other

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RealPlan(Plan):
    """Batched real transform of rank 1-3 with an even last length n (B200 extension; the
    reference's plan API is complex-to-complex only), in numpy's rfftn / irfftn layouts.
    kind "r2c": forward, prod(shape) reals per transform in, prod(shape[:-1]) x (n/2 + 1)
    complex out. kind "c2r": backward, the reverse (imaginary parts of bins 0 and n/2 of every
    last-axis line ignored, as numpy.fft.irfftn does). Out of place only; the normalization
    option scales relative to prod(shape) exactly as for a complex plan of that shape.
    Buffers are float32/float64 and complex64/complex128 tensors (or raw device pointers)."""

    def __init__(self, scalar: str, n, batch_count: int, kind: str, options: plan_options | None = None,
                 device: int | None = None):
        options = options or plan_options()
        if scalar not in ("float", "double"):
            raise SyclfftError(error_code.unsupported_precision, "syclfft supports float and double precision")
        if kind not in ("r2c", "c2r"):
            raise SyclfftError(error_code.invalid_argument, "real transform kind must be 'r2c' or 'c2r'")
        self._lengths = [int(v) for v in n] if isinstance(n, (list, tuple)) else [int(n)]
        self._batch = int(batch_count)
        self._elements = _checked_element_count(self._lengths, self._batch)
        if self._lengths[-1] % 2:
            raise SyclfftError(error_code.invalid_argument, "real transforms need an even last length")
        if options.placement != placement.out_of_place:
            raise SyclfftError(error_code.invalid_argument, "real transforms are out of place")
        self._kind = kind
        self._direction = direction.forward if kind == "r2c" else direction.backward
        self._options = options
        self._double = scalar == "double"
        if options.preferred_provider not in (provider.automatic, provider.b200):
            raise SyclfftError(error_code.provider_unavailable,
                               f"{provider(options.preferred_provider).name} provider is not part of this build")
        torch = _torch()
        if not torch.cuda.is_available():
            raise SyclfftError(error_code.provider_unavailable, "no CUDA device is available")
        self._device = torch.cuda.current_device() if device is None else int(device)
        try:
            self._lib = _provider.load()
        except OSError as e:
            raise SyclfftError(error_code.provider_unavailable, str(e)) from None
        self._api = _provider.provider(self._lib)
        err = ctypes.create_string_buffer(_provider.ERR_CAP)
        if not self._api.supports(self._device, err, _provider.ERR_CAP):
            raise SyclfftError(error_code.provider_unavailable, err.value.decode() or "device not supported")
        cfg = _provider.make_config(self._lengths, self._batch, int(self._direction), self._double, False,
                                    int(options.normalization), options.planning == planning_mode.measure,
                                    self._device)
        self._cfg = cfg
        flags = _provider.CREATE_SYNC
        if options.split_precision and not self._double:
            flags |= _provider.CREATE_SPLIT_BF16
        h = self._lib.syclfft_b200_create_real(ctypes.byref(cfg), _provider.REAL_R2C if kind == "r2c"
                                               else _provider.REAL_C2R, flags, err, _provider.ERR_CAP)
        if not h:
            raise SyclfftError(error_code.planning_failed, err.value.decode() or "B200 plan creation failed")
        self._handle = h
        self._lock = threading.Lock()
        self._last_event = None
        self._last_stream = None
        self._err = ctypes.create_string_buffer(_provider.ERR_CAP)
        self._execute = self._api.execute
        self._bind_fast_path()

    @property
    def kind(self):
        return self._kind

    @property
    def real_dtype(self):
        return _torch().float64 if self._double else _torch().float32

    def _layout(self, name):
        """(dtype, elements) of the input or output buffer."""
        n, b = self._lengths[-1], self._batch
        outer = 1
        for v in self._lengths[:-1]:
            outer *= v
        real = (self.real_dtype, outer * n * b)
        spec = (self.dtype, outer * (n // 2 + 1) * b)
        if self._kind == "r2c":
            return real if name == "input" else spec
        return spec if name == "input" else real

    def _pointer(self, t, name):
        torch = _torch()
        if t is None or (isinstance(t, int) and t == 0):
            raise SyclfftError(error_code.invalid_pointer, f"{name} must be non-null")
        if isinstance(t, int):
            return t
        if not isinstance(t, torch.Tensor) or not t.is_cuda:
            raise SyclfftError(error_code.invalid_pointer, f"{name} is not a device allocation in the plan context")
        if t.device.index != self._device:
            raise SyclfftError(error_code.invalid_pointer, f"{name} lives on another device than the plan")
        dtype, count = self._layout(name)
        if t.dtype != dtype:
            raise SyclfftError(error_code.invalid_argument, f"{name} has dtype {t.dtype}, plan needs {dtype}")
        if not t.is_contiguous() or t.numel() < count:
            raise SyclfftError(error_code.invalid_argument, f"{name} must be contiguous with >= {count} elements")
        return t.data_ptr()

    def move(self) -> "RealPlan":
        other = object.__new__(RealPlan)
        other.__dict__.update(self.__dict__)
        self._handle = None
        return other


def plan_dft_r2c_1d(scalar, n, batch_count=1, options=None, device=None) -> RealPlan:
    """Forward real-to-complex transform(s) of length n: n reals -> n/2 + 1 complex per line."""
    return RealPlan(scalar, n, batch_count, "r2c", options, device)


def plan_dft_r2c(scalar, lengths, batch_count=1, options=None, device=None) -> RealPlan:
    """Forward real-to-complex transform(s) of shape `lengths` (rank 1-3, even last length), as
    numpy.fft.rfftn over the shape's axes."""
    return RealPlan(scalar, list(lengths), batch_count, "r2c", options, device)


def plan_dft_c2r(scalar, lengths, batch_count=1, options=None, device=None) -> RealPlan:
    """Backward complex-to-real transform(s) to shape `lengths`, as numpy.fft.irfftn (times the
    transform size unless a normalization option scales it)."""
    return RealPlan(scalar, list(lengths), batch_count, "c2r", options, device)


def plan_dft_c2r_1d(scalar, n, batch_count=1, options=None, device=None) -> RealPlan:
    """Backward complex-to-real transform(s) of length n: n/2 + 1 complex -> n reals per line."""
    return RealPlan(scalar, n, batch_count, "c2r", options, device)


def plan_many_dft(scalar, lengths, batch_count, dir, options=None, device=None, layout=None) -> Plan:
    """plan_many_dft (syclfft.hpp:90-130); `layout` (B200 extension) gives strided input/output."""
    return Plan(scalar, lengths, batch_count, dir, options, device, layout)


def plan_dft_1d(scalar, n, dir, options=None, device=None) -> Plan:
    return Plan(scalar, [n], 1, dir, options, device)


def plan_dft_2d(scalar, n0, n1, dir, options=None, device=None) -> Plan:
    return Plan(scalar, [n0, n1], 1, dir, options, device)


def plan_dft_3d(scalar, n0, n1, n2, dir, options=None, device=None) -> Plan:
    return Plan(scalar, [n0, n1, n2], 1, dir, options, device)


def query_providers(device: int | None = None):
    """query_providers (sycl.cpp:909-947): status rows for every provider slot."""
    rows = []
    reason = ""
    available = False
    try:
        torch = _torch()
        lib = _provider.load()
        api = _provider.provider(lib)
        if api.abi_version != _provider.ABI_VERSION:
            reason = "B200 provider ABI mismatch"
        elif not torch.cuda.is_available():
            reason = "no CUDA device is available"
        else:
            err = ctypes.create_string_buffer(_provider.ERR_CAP)
            dev = torch.cuda.current_device() if device is None else device
            available = bool(api.supports(dev, err, _provider.ERR_CAP))
            reason = "" if available else err.value.decode()
    except OSError as e:
        reason = str(e)
    rows.append(dict(id=provider.b200, name="b200", built=True, available=available, reason=reason))
    for pid, name, why in ((provider.portable_sycl, "portable_sycl", "not part of this build"),
                           (provider.cufft, "cufft", "not part of this build"),
                           (provider.fftw, "fftw", "not part of this build"),
                           (provider.rocfft, "rocfft", "reserved for a future provider"),
                           (provider.onemkl, "onemkl", "reserved for a future provider")):
        rows.append(dict(id=pid, name=name, built=False, available=False, reason=why))
    return rows
