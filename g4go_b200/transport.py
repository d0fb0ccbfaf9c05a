"""Host-side mirror of G4GO's optical transport interface over the C ABI.

The classes keep the reference's names and meaning so code written against
the C++ interface reads the same here:

  Scene / Material / Surface / Volume / SurfaceBinding
      include/g4go/optical/Scene.hpp:61-164 (volumes are analytic boxes)
  PhotonTransportConfig   include/g4go/optical/PhotonTransportConfig.hpp:26-40
  PhotonTransportBatch    include/g4go/optical/PhotonTransport.hpp:159-163
  PhotonTransportOutput   include/g4go/optical/PhotonTransport.hpp:152-157
  TransportHost           include/g4go/optical/optix/OptiXTransportHost.hpp:10-26
      (PrepareScene -> prepare_scene, EnqueueEmissions -> enqueue_emissions,
       CompleteOldestBatch -> complete_oldest_batch)

Errors are raised with the exception types OptiXTransportHost throws:
ValueError for std::invalid_argument, OverflowError for std::overflow_error,
LogicError for std::logic_error and RuntimeError for CUDA failures
(src/optical/optix/OptiXTransportHost.cpp:47-52,515,524,574-605,655-660,781).
"""
from __future__ import annotations

import collections.abc
import ctypes as C
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _abi

INVALID_ID = _abi.INVALID_ID
EMISSION_DTYPE = _abi.EMISSION_DTYPE
DETECTION_DTYPE = _abi.DETECTION_DTYPE


class LogicError(RuntimeError):
    """std::logic_error: transport queue full or empty, scene rebuild with a pending batch."""


class CapacityError(RuntimeError):
    """An output buffer was too small; the pending batch is kept."""


class NoDeviceError(RuntimeError):
    """No B200 (compute 10.x) device is visible."""


def raise_for_status(status: int, message: str) -> None:
    if status == _abi.OK:
        return
    if status == _abi.ERR_INVALID_ARGUMENT:
        raise ValueError(message)
    if status == _abi.ERR_OVERFLOW:
        raise OverflowError(message)
    if status in (_abi.ERR_LOGIC, _abi.ERR_NO_SCENE):
        raise LogicError(message)
    if status == _abi.ERR_CAPACITY:
        raise CapacityError(message)
    if status == _abi.ERR_NO_DEVICE:
        raise NoDeviceError(message)
    if status == _abi.ERR_UNSUPPORTED:
        raise NotImplementedError(message)
    raise RuntimeError(message)


# ---------------------------------------------------------------------------
# Scene model
# ---------------------------------------------------------------------------

PropertyLike = "tuple[Sequence[float], Sequence[float]] | None"


def _table(value) -> tuple[np.ndarray, np.ndarray] | None:
    if value is None:
        return None
    energy, values = value
    energy = np.ascontiguousarray(energy, dtype=np.float32)
    values = np.ascontiguousarray(values, dtype=np.float32)
    if energy.shape != values.shape or energy.ndim != 1:
        raise ValueError("property tables need matching 1-D energy and value arrays")
    return energy, values


@dataclass
class Material:
    """Material (Scene.hpp:69-76); rayleigh_length_mm is an addition."""

    name: str = ""
    rindex: object = None
    rindex_max: float = 0.0  # 0 -> max of rindex values
    group_velocity_mm_per_ns: object = None
    abs_length_mm: object = None
    rayleigh_length_mm: object = None
    scintillation_spectrum: list = field(default_factory=lambda: [None, None, None])


@dataclass
class Surface:
    """Surface (Scene.hpp:78-92)."""

    name: str = ""
    type: int = _abi.SURFACE_DIELECTRIC_DIELECTRIC
    model: int = _abi.MODEL_UNIFIED
    finish: int = _abi.FINISH_POLISHED
    model_value: float = 1.0
    reflectivity: object = None
    efficiency: object = None
    transmittance: object = None
    rindex: object = None
    specular_lobe: object = None
    specular_spike: object = None
    backscatter: object = None
    surface_roughness: object = None


@dataclass
class Volume:
    """Volume (Scene.hpp:107-120) with an axis-aligned box in world coordinates."""

    name: str = ""
    volume_id: int = INVALID_ID
    material_id: int = INVALID_ID
    parent_volume_id: int = INVALID_ID
    skin_surface_id: int = INVALID_ID
    sensor_id: int = INVALID_ID
    center_mm: tuple = (0.0, 0.0, 0.0)
    half_size_mm: tuple = (1.0, 1.0, 1.0)


@dataclass
class SurfaceBinding:
    """SurfaceBinding (Scene.hpp:122-126): border surface from -> to."""

    from_volume_id: int = INVALID_ID
    to_volume_id: int = INVALID_ID
    surface_id: int = INVALID_ID


class Scene:
    """Scene (Scene.hpp:128-164, Scene.cpp:190-213)."""

    def __init__(self) -> None:
        self.materials: list[Material] = []
        self.surfaces: list[Surface] = []
        self.volumes: list[Volume] = []
        self.surface_bindings: list[SurfaceBinding] = []
        self.world_volume_id: int = INVALID_ID

    def add_material(self, material: Material) -> int:
        self.materials.append(material)
        return len(self.materials) - 1

    def add_surface(self, surface: Surface) -> int:
        self.surfaces.append(surface)
        return len(self.surfaces) - 1

    def add_volume(self, volume: Volume) -> int:
        if volume.volume_id == INVALID_ID:
            volume.volume_id = len(self.volumes)
        self.volumes.append(volume)
        return len(self.volumes) - 1

    def add_surface_binding(self, binding: SurfaceBinding) -> None:
        self.surface_bindings.append(binding)

    def find_volume(self, volume_id: int) -> Volume | None:
        for volume in self.volumes:
            if volume.volume_id == volume_id:
                return volume
        return None

    def to_c(self) -> "CScene":
        return CScene(self)


class CScene:
    """The scene as ABI structures; keeps every array it points into alive."""

    def __init__(self, scene: Scene) -> None:
        self._keep: list = []
        self.materials = (_abi.Material * max(len(scene.materials), 1))()
        for i, m in enumerate(scene.materials):
            self.materials[i].rindex = self._property(m.rindex)
            self.materials[i].rindex_max = float(m.rindex_max)
            self.materials[i].group_velocity_mm_per_ns = self._property(m.group_velocity_mm_per_ns)
            self.materials[i].abs_length_mm = self._property(m.abs_length_mm)
            self.materials[i].rayleigh_length_mm = self._property(m.rayleigh_length_mm)
            spectra = list(m.scintillation_spectrum) + [None] * (3 - len(m.scintillation_spectrum))
            for k in range(3):
                self.materials[i].scintillation_spectrum[k] = self._property(spectra[k])
        self.surfaces = (_abi.Surface * max(len(scene.surfaces), 1))()
        for i, s in enumerate(scene.surfaces):
            target = self.surfaces[i]
            target.type, target.model, target.finish = int(s.type), int(s.model), int(s.finish)
            target.model_value = float(s.model_value)
            for name in (
                "reflectivity", "efficiency", "transmittance", "rindex",
                "specular_lobe", "specular_spike", "backscatter", "surface_roughness",
            ):
                setattr(target, name, self._property(getattr(s, name)))
        self.volumes = (_abi.Volume * max(len(scene.volumes), 1))()
        for i, v in enumerate(scene.volumes):
            target = self.volumes[i]
            target.volume_id = int(v.volume_id)
            target.material_id = int(v.material_id)
            target.parent_volume_id = int(v.parent_volume_id)
            target.skin_surface_id = int(v.skin_surface_id)
            target.sensor_id = int(v.sensor_id)
            for a in range(3):
                target.center_mm[a] = float(v.center_mm[a])
                target.half_size_mm[a] = float(v.half_size_mm[a])
        self.bindings = (_abi.SurfaceBinding * max(len(scene.surface_bindings), 1))()
        for i, b in enumerate(scene.surface_bindings):
            self.bindings[i].from_volume_id = int(b.from_volume_id)
            self.bindings[i].to_volume_id = int(b.to_volume_id)
            self.bindings[i].surface_id = int(b.surface_id)
        self.struct = _abi.Scene()
        self.struct.materials = C.cast(self.materials, C.POINTER(_abi.Material))
        self.struct.material_count = len(scene.materials)
        self.struct.surfaces = C.cast(self.surfaces, C.POINTER(_abi.Surface))
        self.struct.surface_count = len(scene.surfaces)
        self.struct.volumes = C.cast(self.volumes, C.POINTER(_abi.Volume))
        self.struct.volume_count = len(scene.volumes)
        self.struct.bindings = C.cast(self.bindings, C.POINTER(_abi.SurfaceBinding))
        self.struct.binding_count = len(scene.surface_bindings)
        self.struct.world_volume_id = int(scene.world_volume_id)

    def _property(self, value) -> _abi.Property:
        table = _table(value)
        prop = _abi.Property()
        if table is None or table[0].size == 0:
            return prop
        self._keep.extend(table)
        prop.energy_ev = _abi.as_ptr(table[0], C.c_float)
        prop.values = _abi.as_ptr(table[1], C.c_float)
        prop.count = table[0].size
        return prop


# ---------------------------------------------------------------------------
# Config, batch and output
# ---------------------------------------------------------------------------

@dataclass
class PhotonTransportConfig:
    """The transport fields of PhotonTransportConfig plus engine launch knobs."""

    seed: int = 0
    max_bounces_per_photon: int = 4096
    boundary_tolerance_mm: float = 1.0e-4
    precision: str = "fp32"  # "fp32" (FP64 time) or "fp64"
    launch_form: str = "batched"  # "batched" or "plain"
    enable_performance_diagnostics: bool = False
    ordered_detections: bool = True
    hit_capacity: int = 0
    block_size: int = 0
    blocks_per_sm: int = 0
    chunk_photons: int = 0
    use_cuda_graph: bool = True
    record_photon_fates: bool = False
    # batched FP32: 0/1 separate generation kernel for batches of >= 2^24 photons,
    # 2 generation inside the loop, 3 separate generation kernel at any size
    generation_pass: int = 0
    wave_photons: int = 0  # most photons per generation-pass wave (0: sized by free device memory, <= 2^28)
    device: int = -1

    def to_c(self) -> _abi.Config:
        config = _abi.Config()
        config.abi_version = _abi.ABI_VERSION
        config.device = int(self.device)
        config.seed = int(self.seed) & 0xFFFFFFFFFFFFFFFF
        config.max_bounces_per_photon = int(self.max_bounces_per_photon)
        config.boundary_tolerance_mm = float(self.boundary_tolerance_mm)
        precisions = {"fp32": _abi.PRECISION_FP32, "fp64": _abi.PRECISION_FP64}
        forms = {"batched": _abi.FORM_BATCHED, "plain": _abi.FORM_PLAIN}
        if self.precision not in precisions or self.launch_form not in forms:
            raise ValueError("precision must be fp32|fp64 and launch_form batched|plain")
        config.precision = precisions[self.precision]
        config.launch_form = forms[self.launch_form]
        config.enable_performance_diagnostics = int(bool(self.enable_performance_diagnostics))
        config.ordered_detections = int(bool(self.ordered_detections))
        config.hit_capacity = int(self.hit_capacity)
        config.block_size = int(self.block_size)
        config.blocks_per_sm = int(self.blocks_per_sm)
        config.chunk_photons = int(self.chunk_photons)
        config.use_cuda_graph = int(bool(self.use_cuda_graph))
        config.record_photon_fates = int(bool(self.record_photon_fates))
        config.generation_pass = int(self.generation_pass)
        config.wave_photons = int(self.wave_photons)
        return config


@dataclass
class PhotonTransportBatch:
    """PhotonTransportBatch: gensteps, the batch's event IDs, and each genstep's event index."""

    emissions: np.ndarray
    event_ids: np.ndarray
    emission_event_indices: np.ndarray

    def __post_init__(self) -> None:
        self.emissions = np.ascontiguousarray(self.emissions, dtype=EMISSION_DTYPE)
        self.event_ids = np.ascontiguousarray(self.event_ids, dtype=np.uint32)
        self.emission_event_indices = np.ascontiguousarray(self.emission_event_indices, dtype=np.uint32)

    @property
    def photon_count(self) -> int:
        return int(self.emissions["photon_count"].sum(dtype=np.uint64))

    def photon_slice(self, begin: int, end: int, ends: np.ndarray | None = None):
        """The gensteps that hold flattened photon slots [begin, end) as a batch
        of their own, with the slots' range inside it: (batch, (b, e)). Every
        photon keeps its event ID and photon ID, and so its random numbers and
        its history. `ends` (the cumulative photon counts, int64) may be passed
        to save recomputing it for many slices."""
        if ends is None:
            ends = np.cumsum(self.emissions["photon_count"], dtype=np.int64)
        total = int(ends[-1]) if ends.size else 0
        if not 0 <= begin < end <= total:
            raise ValueError(f"photon slice [{begin}, {end}) outside [0, {total})")
        first = int(np.searchsorted(ends, begin, side="right"))
        last = int(np.searchsorted(ends, end - 1, side="right")) + 1
        events, local = np.unique(self.emission_event_indices[first:last], return_inverse=True)
        part = PhotonTransportBatch(self.emissions[first:last], self.event_ids[events], local.astype(np.uint32))
        offset = int(ends[first - 1]) if first > 0 else 0
        return part, (begin - offset, end - offset)


STAT_FIELDS = (
    "valid_fields", "generated_count", "captured_count", "detected_count", "absorbed_count", "escaped_count",
    "truncated_count", "max_bounce_count", "invalid_state_count", "zero_step_count", "transport_time_ms",
)
PERF_FIELDS = tuple(name for name, _ in _abi.Performance._fields_)


def _stats_dict(stats: _abi.Statistics) -> dict:
    return {name: getattr(stats, name) for name in STAT_FIELDS}


class EventStatisticsList(collections.abc.Sequence):
    """A completed batch's per-event statistics, [(event_id, statistics dict)]
    in batch order. The engine's records stay in one numpy array until the
    first read, which converts every event at once, column by column; a caller
    that never reads them pays nothing per event (building 50,000 dicts takes
    longer than a tenth of that batch's transport)."""

    def __init__(self, records: np.ndarray):
        self._records = records
        self._events: list | None = None

    def _list(self) -> list:
        if self._events is None:
            statistics = self._records["statistics"]
            columns = [statistics[name].tolist() for name in STAT_FIELDS]
            self._events = [(event_id, dict(zip(STAT_FIELDS, values)))
                            for event_id, values in zip(self._records["event_id"].tolist(), zip(*columns))]
        return self._events

    def __len__(self) -> int:
        return int(self._records.shape[0])

    def __getitem__(self, index):
        return self._list()[index]

    def __iter__(self):
        return iter(self._list())

    def __eq__(self, other):
        if isinstance(other, (EventStatisticsList, list, tuple)):
            return self._list() == list(other)
        return NotImplemented

    def __repr__(self) -> str:
        return f"EventStatisticsList({self._list()!r})"


def _check_detection_buffer(buffer) -> None:
    """A caller's detection buffer must take g4b_complete's records in place:
    the engine writes `capacity` 48-byte records from its first byte."""
    if not isinstance(buffer, np.ndarray) or buffer.ndim != 1:
        raise ValueError("detections_out must be a one-dimensional numpy array")
    if buffer.dtype != DETECTION_DTYPE:
        raise ValueError(f"detections_out must have the detection record dtype, not {buffer.dtype}")
    if not buffer.flags.c_contiguous:
        raise ValueError("detections_out must be C-contiguous (a strided view would be written across)")
    if not buffer.flags.writeable:
        raise ValueError("detections_out must be writeable")


def _event_statistics(records, count: int) -> EventStatisticsList:
    return EventStatisticsList(np.ctypeslib.as_array(records)[:count])


@dataclass
class PhotonTransportOutput:
    detections: np.ndarray
    statistics: dict
    performance: dict
    event_statistics: Sequence  # [(event_id, statistics dict)], an EventStatisticsList


def statistic_field_bit(field_index: int) -> int:
    return 1 << field_index


# ---------------------------------------------------------------------------
# TransportHost (OptiXTransportHost)
# ---------------------------------------------------------------------------

class TransportHost:
    """OptiXTransportHost over the B200 engine: one pending batch at a time."""

    def __init__(self, config: PhotonTransportConfig | None = None) -> None:
        self._lib = _abi.load()
        self.config = config or PhotonTransportConfig()
        handle = C.c_void_p()
        status = self._lib.g4b_create(C.byref(self.config.to_c()), C.byref(handle))
        if status != _abi.OK:
            raise_for_status(status, self._lib.g4b_last_error(None).decode())
        self._handle = handle
        self._scene_ref: Scene | None = None
        self._c_scene: CScene | None = None
        self._pending_batch: PhotonTransportBatch | None = None
        self._last_batch: PhotonTransportBatch | None = None

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_handle", None):
            self._lib.g4b_destroy(self._handle)
            self._handle = None

    def __enter__(self) -> "TransportHost":
        return self

    def __exit__(self, *exc) -> None:
        self.close()

    def __del__(self) -> None:
        try:
            self.close()
        except Exception:
            pass

    def _check(self, status: int) -> None:
        if status != _abi.OK:
            raise_for_status(status, self._lib.g4b_last_error(self._handle).decode())

    # -- the reference interface -------------------------------------------
    def prepare_scene(self, scene: Scene) -> None:
        """PrepareScene: rebuilds when a different Scene object is passed (OptiXTransportHost.cpp:511-519)."""
        if scene is self._scene_ref:
            return
        c_scene = scene.to_c()
        self._check(self._lib.g4b_set_scene(self._handle, C.byref(c_scene.struct)))
        self._scene_ref = scene
        self._c_scene = c_scene

    def enqueue_emissions(self, scene: Scene, batch: PhotonTransportBatch) -> None:
        """EnqueueEmissions (OptiXTransportHost.cpp:521-777)."""
        self.prepare_scene(scene)
        emissions = batch.emissions
        self._check(
            self._lib.g4b_enqueue(
                self._handle,
                emissions.ctypes.data_as(C.c_void_p),
                emissions.shape[0],
                _abi.as_ptr(batch.event_ids, C.c_uint32),
                batch.event_ids.shape[0],
                _abi.as_ptr(batch.emission_event_indices, C.c_uint32),
            )
        )
        self._pending_batch = batch
        self._last_batch = batch

    def relaunch(self) -> None:
        """Re-runs the last enqueued batch on its device-resident copy."""
        self._check(self._lib.g4b_relaunch(self._handle))

    def query_oldest(self) -> tuple[int, int]:
        detections = C.c_uint64()
        events = C.c_uint32()
        self._check(self._lib.g4b_query_oldest(self._handle, C.byref(detections), C.byref(events)))
        return int(detections.value), int(events.value)

    def complete_oldest_batch(self, detections_out: np.ndarray | None = None,
                              counts_only: bool = False) -> PhotonTransportOutput:
        """CompleteOldestBatch (OptiXTransportHost.cpp:779-883).

        counts_only: return statistics without copying the detections back
        (they stay in device memory).
        detections_out: a C-contiguous, writeable array of DETECTION_DTYPE
        records (ValueError otherwise): the engine writes 48-byte records into
        it by address."""
        if detections_out is not None:
            _check_detection_buffer(detections_out)
        if detections_out is not None and not counts_only and self._pending_batch is not None:
            # a caller buffer: complete at once, without first waiting for the
            # counts, so that a multi-wave batch's detections stream into it
            # while its later waves still run; too small -> the counts first
            events = int(self._pending_batch.event_ids.shape[0])
            done = self._complete_into(detections_out, detections_out.shape[0], events)
            if done is not None:
                return done
        count, events = self.query_oldest()
        if counts_only:
            detections_out = np.empty(0, dtype=DETECTION_DTYPE)
        elif detections_out is None or detections_out.shape[0] < count:
            detections_out = np.empty(count, dtype=DETECTION_DTYPE)
        event_stats = (_abi.EventStatistics * max(events, 1))()
        output = _abi.Output()
        output.detections = detections_out.ctypes.data_as(C.c_void_p) if (count and not counts_only) else None
        output.detection_capacity = 0 if counts_only else detections_out.shape[0]
        output.event_statistics = C.cast(event_stats, C.POINTER(_abi.EventStatistics))
        output.event_capacity = events
        self._check(self._lib.g4b_complete(self._handle, C.byref(output)))
        self._pending_batch = None
        perf = {name: getattr(output.performance, name) for name in PERF_FIELDS}
        event_list = _event_statistics(event_stats, events)
        return PhotonTransportOutput(
            detections=detections_out[: 0 if counts_only else output.detection_count],
            statistics=_stats_dict(output.statistics),
            performance=perf,
            event_statistics=event_list,
        )

    def _complete_into(self, detections_out: np.ndarray, capacity: int, events: int):
        """g4b_complete into the caller's buffer; None if it is too small (the batch stays pending)."""
        event_stats = (_abi.EventStatistics * max(events, 1))()
        output = _abi.Output()
        output.detections = detections_out.ctypes.data_as(C.c_void_p)
        output.detection_capacity = capacity
        output.event_statistics = C.cast(event_stats, C.POINTER(_abi.EventStatistics))
        output.event_capacity = events
        status = self._lib.g4b_complete(self._handle, C.byref(output))
        if status == _abi.ERR_CAPACITY:
            return None
        self._check(status)
        self._pending_batch = None
        perf = {name: getattr(output.performance, name) for name in PERF_FIELDS}
        event_list = _event_statistics(event_stats, output.event_count)
        return PhotonTransportOutput(
            detections=detections_out[: output.detection_count],
            statistics=_stats_dict(output.statistics),
            performance=perf,
            event_statistics=event_list,
        )

    # -- engine extras -------------------------------------------------------
    @property
    def stream(self) -> int:
        pointer = C.c_void_p()
        self._check(self._lib.g4b_get_stream(self._handle, C.byref(pointer)))
        return int(pointer.value or 0)

    def photon_fates(self) -> tuple[np.ndarray, np.ndarray]:
        count = C.c_uint64()
        status = self._lib.g4b_photon_fates(self._handle, None, None, 0, C.byref(count))
        if status not in (_abi.OK, _abi.ERR_CAPACITY):
            self._check(status)
        n = int(count.value)
        fate = np.empty(n, dtype=np.uint32)
        time = np.empty(n, dtype=np.float64)
        self._check(
            self._lib.g4b_photon_fates(
                self._handle, _abi.as_ptr(fate, C.c_uint32), _abi.as_ptr(time, C.c_double), n, C.byref(count)
            )
        )
        return fate, time

    PARAMETERS = ("rindex", "abs_length_mm", "reflectivity", "decay_time_ns")

    def gradients(self, rindex_material: int = INVALID_ID, abs_length_material: int = INVALID_ID,
                  reflectivity_surface: int = INVALID_ID, edge_band_mm: float | None = None,
                  edge_index_window: float | None = None) -> dict:
        """d(detected)/d theta and d(mean arrival time)/d theta for the last completed batch.

        The index derivative's boundary term of box edges is estimated in a
        window of half width edge_band_mm (None: the library's 0.1 mm; 0: no
        boundary term), widened for fast edges to the distance they move over
        +-edge_index_window in n when that is given (lower variance, a bias
        growing with it)."""
        band = 0.0 if edge_band_mm is None else (float(edge_band_mm) if edge_band_mm > 0 else -1.0)
        window = float(edge_index_window) if edge_index_window else 0.0
        request = _abi.GradientRequest(rindex_material, abs_length_material, reflectivity_surface, band, window)
        result = _abi.Gradients()
        self._check(self._lib.g4b_gradients(self._handle, C.byref(request), C.byref(result)))
        return {
            "detected": int(result.detected),
            "mean_time_ns": float(result.mean_time_ns),
            "d_detected": dict(zip(self.PARAMETERS, list(result.d_detected))),
            "d_mean_time_ns": dict(zip(self.PARAMETERS, list(result.d_mean_time_ns))),
            "replay_mismatches": int(result.replay_mismatches),
            "kernel_ms": float(result.kernel_ms),
        }

    def autotune(self, block_sizes: Sequence[int] = (), chunk_sizes: Sequence[int] = (), repeats: int = 2) -> dict:
        blocks = np.ascontiguousarray(block_sizes, dtype=np.uint32)
        chunks = np.ascontiguousarray(chunk_sizes, dtype=np.uint32)
        result = _abi.TuneResult()
        self._check(
            self._lib.g4b_autotune(
                self._handle,
                _abi.as_ptr(blocks, C.c_uint32) if blocks.size else None,
                blocks.size,
                _abi.as_ptr(chunks, C.c_uint32) if chunks.size else None,
                chunks.size,
                repeats,
                C.byref(result),
            )
        )
        return {name: getattr(result, name) for name, _ in _abi.TuneResult._fields_}


# ---------------------------------------------------------------------------
# Device-evaluated boundary functions and math (for unit checks on the GPU)
# ---------------------------------------------------------------------------

def _lib():
    return _abi.load()


def _handleless(status: int) -> None:
    if status != _abi.OK:
        raise_for_status(status, _lib().g4b_last_error(None).decode())


def eval_fresnel(direction, polarization, normal, index_from, index_to, precision: str = "fp32", device: int = -1):
    """ComputeFresnel on the GPU: returns an (n, 14) array."""
    d = np.ascontiguousarray(direction, dtype=np.float64).reshape(-1, 3)
    p = np.ascontiguousarray(polarization, dtype=np.float64).reshape(-1, 3)
    nrm = np.ascontiguousarray(normal, dtype=np.float64).reshape(-1, 3)
    n1 = np.ascontiguousarray(index_from, dtype=np.float64).reshape(-1)
    n2 = np.ascontiguousarray(index_to, dtype=np.float64).reshape(-1)
    out = np.empty((d.shape[0], 14), dtype=np.float64)
    _handleless(
        _lib().g4b_eval_fresnel(
            device, _abi.PRECISION_FP64 if precision == "fp64" else _abi.PRECISION_FP32, d.shape[0],
            _abi.as_ptr(d, C.c_double), _abi.as_ptr(p, C.c_double), _abi.as_ptr(nrm, C.c_double),
            _abi.as_ptr(n1, C.c_double), _abi.as_ptr(n2, C.c_double), _abi.as_ptr(out, C.c_double),
        )
    )
    return out


def eval_lambertian(normal, radial, azimuth, precision: str = "fp32", device: int = -1):
    nrm = np.ascontiguousarray(normal, dtype=np.float64).reshape(-1, 3)
    r = np.ascontiguousarray(radial, dtype=np.float64).reshape(-1)
    a = np.ascontiguousarray(azimuth, dtype=np.float64).reshape(-1)
    out = np.empty((nrm.shape[0], 3), dtype=np.float64)
    _handleless(
        _lib().g4b_eval_lambertian(
            device, _abi.PRECISION_FP64 if precision == "fp64" else _abi.PRECISION_FP32, nrm.shape[0],
            _abi.as_ptr(nrm, C.c_double), _abi.as_ptr(r, C.c_double), _abi.as_ptr(a, C.c_double),
            _abi.as_ptr(out, C.c_double),
        )
    )
    return out


def eval_math(kind: str, x, device: int = -1):
    kinds = {"log": 0, "exp": 1, "sincos_turn": 2}
    values = np.ascontiguousarray(x, dtype=np.float32).reshape(-1)
    n = values.size
    out = np.empty(2 * n if kind == "sincos_turn" else n, dtype=np.float32)
    _handleless(_lib().g4b_eval_math(device, kinds[kind], n, _abi.as_ptr(values, C.c_float), _abi.as_ptr(out, C.c_float)))
    if kind == "sincos_turn":
        return out[:n], out[n:]
    return out


def eval_uniform(seed: int, keys, bounce, process, draw, device: int = -1):
    k = np.ascontiguousarray(keys, dtype=np.uint64)
    b = np.ascontiguousarray(bounce, dtype=np.uint32)
    pr = np.ascontiguousarray(process, dtype=np.uint32)
    dr = np.ascontiguousarray(draw, dtype=np.uint32)
    out = np.empty(k.size, dtype=np.float32)
    _handleless(
        _lib().g4b_eval_uniform(
            device, k.size, seed, _abi.as_ptr(k, C.c_uint64), _abi.as_ptr(b, C.c_uint32),
            _abi.as_ptr(pr, C.c_uint32), _abi.as_ptr(dr, C.c_uint32), _abi.as_ptr(out, C.c_float),
        )
    )
    return out
