"""The C ABI without a GPU: the library loads, exports every declared symbol,
its record layouts match the reference's, and it fails loudly with no device."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions(headers=None):
    names = set()
    for header in HEADERS if headers is None else headers:
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for match in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(g4b_\w+)\s*\(", text, flags=re.M):
            names.add(match.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported(engine_lib):
    """libg4b.so exports what g4b.h and g4b_scheduler.h declare; the genstep
    source (g4b_synth.h) is a library of its own, and the engine carries none
    of it."""
    from g4go_b200 import _abi

    synth_header = [h for h in HEADERS if h.name == "g4b_synth.h"]
    names = declared_functions([h for h in HEADERS if h.name != "g4b_synth.h"])
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(engine_lib, n)]
    assert not missing, missing
    assert set(names) == set(_abi.SIGNATURES), "the ctypes binding must cover exactly the declared symbols"
    synth_names = declared_functions(synth_header)
    synth = _abi.load_synth()
    assert synth_names and not [n for n in synth_names if not hasattr(synth, n)]
    assert set(synth_names) == set(_abi.SYNTH_SIGNATURES)
    assert not [n for n in synth_names if hasattr(engine_lib, n)]


def test_record_layouts_match_the_reference(tmp_path):
    """sizeof/offsetof from a C compiler against the ctypes and numpy views."""
    from g4go_b200 import _abi

    program = tmp_path / "layout.c"
    program.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "g4b.h"\n#include "g4b_synth.h"\n#include "g4b_scheduler.h"\n'
        "int main(void){\n"
        ' printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
        " sizeof(g4b_optical_emission), sizeof(g4b_photon_detection), sizeof(g4b_config), sizeof(g4b_property),"
        " sizeof(g4b_material), sizeof(g4b_surface), sizeof(g4b_volume), sizeof(g4b_scene), sizeof(g4b_statistics),"
        " sizeof(g4b_event_statistics), sizeof(g4b_performance), sizeof(g4b_output), sizeof(g4b_synth_params),"
        " offsetof(g4b_optical_emission, type));\n"
        ' printf("%zu %zu %zu %zu\\n", offsetof(g4b_optical_emission, event_id),'
        " offsetof(g4b_optical_emission, photon_count), offsetof(g4b_photon_detection, sensor_id),"
        " offsetof(g4b_config, hit_capacity));\n"
        ' printf("%zu %zu %zu %zu\\n", sizeof(g4b_scheduler_config), sizeof(g4b_batch_statistics),'
        " sizeof(g4b_transport_ops), offsetof(g4b_batch_statistics, performance));\n"
        " return 0; }\n"
    )
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(program), "-o", str(exe)], check=True)
    first, second, third = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines()
    sizes = list(map(int, first.split()))
    offsets = list(map(int, second.split()))
    assert sizes[0] == 128 and sizes[1] == 48  # PhotonTransport.hpp:177-178
    expected = [_abi.EMISSION_DTYPE.itemsize, _abi.DETECTION_DTYPE.itemsize, C.sizeof(_abi.Config),
                C.sizeof(_abi.Property), C.sizeof(_abi.Material), C.sizeof(_abi.Surface), C.sizeof(_abi.Volume),
                C.sizeof(_abi.Scene), C.sizeof(_abi.Statistics), C.sizeof(_abi.EventStatistics),
                C.sizeof(_abi.Performance), C.sizeof(_abi.Output), C.sizeof(_abi.SynthParams),
                _abi.EMISSION_DTYPE.fields["type"][1]]
    assert sizes == expected
    # OpticalEmission field offsets (PhotonTransport.hpp:40-69): eventID at 88, photonCount at 96.
    assert offsets[0] == 88 == _abi.EMISSION_DTYPE.fields["event_id"][1]
    assert offsets[1] == 96 == _abi.EMISSION_DTYPE.fields["photon_count"][1]
    assert offsets[2] == 40 == _abi.DETECTION_DTYPE.fields["sensor_id"][1]
    assert offsets[3] == _abi.Config.hit_capacity.offset
    # the batch scheduler's records (include/g4b_scheduler.h)
    assert list(map(int, third.split())) == [C.sizeof(_abi.SchedulerConfig), C.sizeof(_abi.BatchStatistics),
                                             C.sizeof(_abi.TransportOps), _abi.BatchStatistics.performance.offset]


def test_cpp_shim_compiles(tmp_path):
    """The header-only C++ drop-in (OptiXTransportHost signatures over the C ABI) builds and links."""
    source = tmp_path / "shim.cpp"
    source.write_text('#include "g4b_transport_host.hpp"\nint main(){ return 0; }\n')
    from g4go_b200 import _abi

    library = _abi.library_path()
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), str(source),
                    str(library), "-o", str(tmp_path / "shim")], check=True)


def test_engine_fails_loudly_without_a_device(engine_lib):
    from conftest import gpu_available
    from g4go_b200 import NoDeviceError, PhotonTransportConfig, TransportHost

    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(NoDeviceError):
        TransportHost(PhotonTransportConfig())


def test_config_rejects_bad_abi_version(engine_lib):
    from g4go_b200 import _abi

    config = _abi.Config()
    config.abi_version = 999
    handle = C.c_void_p()
    status = engine_lib.g4b_create(C.byref(config), C.byref(handle))
    assert status == _abi.ERR_INVALID_ARGUMENT
    assert b"abi_version" in engine_lib.g4b_last_error(None)


def test_synthetic_gensteps_are_seeded_and_well_formed(engine_lib):
    from g4go_b200 import scenes

    a = scenes.workload("batched", event_count=300, seed=5)
    b = scenes.workload("batched", event_count=300, seed=5)
    c = scenes.electron_gensteps(300, **{k: v for k, v in scenes.WORKLOADS["batched"].items() if k != "event_count"},
                                 seed=5, threads=1)
    assert a.emissions.tobytes() == b.emissions.tobytes() == c.emissions.tobytes()
    assert np.all(a.emissions["event_id"] == a.event_ids[a.emission_event_indices])
    assert set(np.unique(a.emissions["type"])) <= {1, 2}
    # photon IDs within an event are consecutive from 0
    for event in range(5):
        rows = a.emissions[a.emission_event_indices == event]
        starts = rows["first_photon_id"]
        assert starts[0] == 0
        assert np.all(starts[1:] == starts[:-1] + rows["photon_count"][:-1])
    # uneven events: tens to ~1e5 photons
    per_event = np.bincount(a.emission_event_indices, weights=a.emissions["photon_count"], minlength=300)
    assert per_event.max() > 50 * max(per_event.min(), 1)


def test_event_statistics_read_as_the_list_of_the_records():
    """complete_oldest_batch returns g4b_event_statistics records as an
    EventStatisticsList: the [(event_id, statistics dict)] list, in batch order,
    built on first read with the same Python types as a field-by-field read."""
    from g4go_b200 import _abi, transport

    records = (_abi.EventStatistics * 5)()
    for i in range(5):
        records[i].event_id = 100 + 7 * i
        records[i].statistics.valid_fields = 0x3ff
        records[i].statistics.detected_count = 2 ** 40 + i
        records[i].statistics.transport_time_ms = 0.25 * i
    expected = [(int(r.event_id), transport._stats_dict(r.statistics)) for r in records[:4]]
    view = transport._event_statistics(records, 4)
    assert len(view) == 4
    assert view == expected and expected == list(view)
    assert view[0] == expected[0] and view[-1][0] == 121 and view[1:3] == expected[1:3]
    assert [e for e, _ in view] == [100, 107, 114, 121]
    assert type(view[3][1]["detected_count"]) is int and type(view[3][1]["transport_time_ms"]) is float
    assert view == transport._event_statistics(records, 4)
    assert view != transport._event_statistics(records, 5)
    assert transport._event_statistics(records, 0) == []


def test_caller_detection_buffers_are_checked_before_the_engine_writes():
    """complete_oldest_batch(detections_out=...) hands the array's address to
    g4b_complete, which writes 48-byte records: a wrong dtype, a strided view or
    a read-only array must be refused before any engine call."""
    import numpy as np

    from g4go_b200 import transport

    host = object.__new__(transport.TransportHost)  # no device here: the check comes first
    good = np.empty(8, dtype=transport.DETECTION_DTYPE)
    transport._check_detection_buffer(good)
    readonly = np.empty(8, dtype=transport.DETECTION_DTYPE)
    readonly.flags.writeable = False
    for bad in (np.empty(8 * 48, dtype=np.uint8), np.empty(16, dtype=transport.DETECTION_DTYPE)[::2],
                readonly, np.empty((2, 4), dtype=transport.DETECTION_DTYPE)):
        with pytest.raises(ValueError):
            host.complete_oldest_batch(detections_out=bad)


# the ctypes view of every record the C ABI passes, and the C struct it mirrors
CTYPES_RECORDS = {
    "Config": "g4b_config", "Property": "g4b_property", "Material": "g4b_material", "Surface": "g4b_surface",
    "Volume": "g4b_volume", "SurfaceBinding": "g4b_surface_binding", "Scene": "g4b_scene",
    "Statistics": "g4b_statistics", "EventStatistics": "g4b_event_statistics", "Performance": "g4b_performance",
    "Output": "g4b_output", "TuneResult": "g4b_tune_result", "GradientRequest": "g4b_gradient_request",
    "Gradients": "g4b_gradient_result", "SchedulerConfig": "g4b_scheduler_config",
    "BatchStatistics": "g4b_batch_statistics", "TransportOps": "g4b_transport_ops", "SynthParams": "g4b_synth_params",
}


def test_every_ctypes_field_sits_where_the_header_puts_it(tmp_path):
    """Size and the offset of every field of each ctypes record, from a C
    compiler on include/*.h, so that a field added to a header without its
    ctypes mirror (or the other way round) fails here, not on a GPU."""
    from g4go_b200 import _abi

    checks = []
    for py_name, c_name in CTYPES_RECORDS.items():
        record = getattr(_abi, py_name)
        checks.append((f"sizeof({c_name})", C.sizeof(record), py_name))
        for field in record._fields_:
            checks.append((f"offsetof({c_name}, {field[0]})", getattr(record, field[0]).offset, f"{py_name}.{field[0]}"))
    program = tmp_path / "fields.c"
    body = "".join(f' printf("%zu\\n", (size_t){expr});\n' for expr, _, _ in checks)
    program.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "g4b.h"\n#include "g4b_synth.h"\n'
                       '#include "g4b_scheduler.h"\nint main(void){\n' + body + " return 0; }\n")
    exe = tmp_path / "fields"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(program), "-o", str(exe)], check=True)
    values = list(map(int, subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()))
    mismatches = [(what, c, py) for (_, py, what), c in zip(checks, values) if c != py]
    assert not mismatches, mismatches
