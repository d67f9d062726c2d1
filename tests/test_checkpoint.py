"""CPU: checkpoint interchange in the reference's restart format.

The metadata cases mirror the reference's tests/checkpoint_config_tests.cpp
(same compatibility records and expectations); the file cases check the
state file byte for byte against the layout of src/Simulation.cpp:1571-1580,
read back here with plain struct unpacking, and the load-side failures of
src/Simulation.cpp:1477-1538."""
import json
import os
import struct

import numpy as np
import pytest

from theseus_b200.checkpoint import (CheckpointCompatibility, CheckpointConfig, load_checkpoint,
                                     save_checkpoint)

EXPECTED = CheckpointCompatibility(2, 3, 2, 4, 8, 576, 9216, False)


def compat(**kw):
    d = dict(EXPECTED.__dict__)
    d.update(kw)
    return CheckpointCompatibility(**d)


def test_checkpoints_default_to_disabled():
    cfg = CheckpointConfig.from_runtime({}, "output")
    assert not cfg.load and not cfg.save
    assert cfg.interval == pytest.approx(0.01, abs=1e-15)
    assert cfg.directory == os.path.join("output", "Checkpoints")


def test_checkpoint_paths_are_constructed_consistently():
    cfg = CheckpointConfig.from_runtime({"checkpoint_load": True, "checkpoint_save": True,
                                         "checkpoint_cycle": 12, "checkpoint_dt": 0.25,
                                         "checkpoints_folder": "restart-data"}, "results")
    assert cfg.load and cfg.save and cfg.cycle == 12
    assert cfg.metadata_file(12) == "results/restart-data/Cycle12/checkpoint_cycle_12.json"
    assert cfg.rank_file(12, 3) == "results/restart-data/Cycle12/checkpoint_cycle_12.00000003.chk"


def test_checkpoint_loading_requires_a_positive_cycle():
    with pytest.raises(ValueError, match="checkpoint_cycle"):
        CheckpointConfig.from_runtime({"checkpoint_load": True}, ".")


def test_enabled_checkpoints_require_a_positive_interval():
    with pytest.raises(ValueError, match="checkpoint_dt"):
        CheckpointConfig.from_runtime({"checkpoint_save": True, "checkpoint_dt": 0.0}, ".")


def test_current_checkpoint_metadata_validates_compatibility():
    md = CheckpointConfig.metadata(0.1, 10, EXPECTED)
    assert md["format_version"] == 2
    assert md["state_representation"] == "conservative"
    assert md["geometry"] == "cartesian"
    assert md["state_format"] == "raw_vector_v1"
    assert md["time"] == 0.1 and md["cycle"] == 10
    assert CheckpointConfig.validate_metadata(md, EXPECTED) is True


def test_checkpoint_metadata_rejects_an_incompatible_mpi_layout():
    md = CheckpointConfig.metadata(0.1, 10, EXPECTED)
    with pytest.raises(ValueError, match="mpi_ranks"):
        CheckpointConfig.validate_metadata(md, compat(mpi_ranks=4))


@pytest.mark.parametrize("field", ["order", "dimension", "num_equations", "global_elements",
                                   "global_dofs"])
def test_checkpoint_metadata_rejects_each_discretisation_mismatch(field):
    md = CheckpointConfig.metadata(0.1, 10, EXPECTED)
    with pytest.raises(ValueError, match=f"{field} differs"):
        CheckpointConfig.validate_metadata(md, compat(**{field: getattr(EXPECTED, field) + 1}))


def test_checkpoint_metadata_rejects_another_real_size():
    md = CheckpointConfig.metadata(0.1, 10, EXPECTED)
    with pytest.raises(ValueError, match="floating-point representation"):
        CheckpointConfig.validate_metadata(md, compat(real_bytes=4))


def test_legacy_checkpoint_metadata_remains_loadable():
    assert CheckpointConfig.validate_metadata({"time": 0.1, "cycle": 10}, EXPECTED) is False


def test_axisymmetric_checkpoint_records_conservative_state_semantics():
    ax = compat(axisymmetric=True)
    md = CheckpointConfig.metadata(0.1, 10, ax)
    assert md["state_representation"] == "conservative" and md["geometry"] == "axisymmetric"
    assert CheckpointConfig.validate_metadata(md, ax) is True


def test_axisymmetric_restart_rejects_ambiguous_ru_checkpoint_metadata():
    ax = compat(axisymmetric=True)
    md = CheckpointConfig.metadata(0.1, 10, ax)
    md["format_version"] = 1
    del md["state_representation"], md["geometry"]
    with pytest.raises(ValueError, match="U or rU"):
        CheckpointConfig.validate_metadata(md, ax)


def test_checkpoint_geometry_must_match_current_run():
    md = CheckpointConfig.metadata(0.1, 10, EXPECTED)
    with pytest.raises(ValueError, match="geometry"):
        CheckpointConfig.validate_metadata(md, compat(axisymmetric=True))


def test_unsupported_versions_and_formats_are_rejected():
    md = CheckpointConfig.metadata(0.1, 10, EXPECTED)
    with pytest.raises(ValueError, match="format version"):
        CheckpointConfig.validate_metadata(dict(md, format_version=3), EXPECTED)
    with pytest.raises(ValueError, match="state format"):
        CheckpointConfig.validate_metadata(dict(md, state_format="hdf5"), EXPECTED)
    with pytest.raises(ValueError, match="state representation"):
        CheckpointConfig.validate_metadata(dict(md, state_representation="primitive"), EXPECTED)
    with pytest.raises(ValueError, match="not a JSON object"):
        CheckpointConfig.validate_metadata("[1, 2]", EXPECTED)


def test_metadata_time_round_trips_exactly():
    for t in (0.1, 1.0, 1e-300, 123456.789, 2.0 / 3.0, 0.0):
        md = CheckpointConfig.metadata(t, 3, EXPECTED)
        assert md["time"] == t


def test_state_file_layout_and_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    c = compat(mpi_ranks=1, global_dofs=4 * 576 * 16)
    u = rng.standard_normal((4, 576, 16))
    d = str(tmp_path / "Checkpoints")
    save_checkpoint(d, 7, u, 0.125, c)
    cfg = CheckpointConfig(directory=d)
    raw = open(cfg.rank_file(7, 0), "rb").read()
    head = b"THESEUS_CHECKPOINT_RAW_V1\n"
    assert raw.startswith(head)
    (n,) = struct.unpack_from("<Q", raw, len(head))
    assert n == u.size and len(raw) == len(head) + 8 + 8 * n
    assert np.array_equal(np.frombuffer(raw, "<f8", offset=len(head) + 8), u.reshape(-1))
    md = json.load(open(cfg.metadata_file(7)))
    assert md["time"] == 0.125 and md["cycle"] == 7 and md["global_dofs"] == u.size
    t, back = load_checkpoint(d, 7, c, shape=u.shape)
    assert t == 0.125 and np.array_equal(back, u)


def test_rank_files_are_per_rank(tmp_path):
    d = str(tmp_path)
    c = compat(mpi_ranks=2, global_dofs=20)
    for r in range(2):
        save_checkpoint(d, 4, np.full(10, float(r)), 0.5, c, rank=r, write_metadata=(r == 0))
    for r in range(2):
        t, s = load_checkpoint(d, 4, c, rank=r)
        assert t == 0.5 and np.all(s == r) and s.size == 10


def test_load_failures_follow_the_reference(tmp_path):
    d = str(tmp_path)
    c = compat(mpi_ranks=1, global_dofs=12)
    save_checkpoint(d, 5, np.arange(12.0), 1.5, c)
    cfg = CheckpointConfig(directory=d)
    with pytest.raises(OSError, match="Failed to open checkpoint metadata"):
        load_checkpoint(d, 6, c)
    with pytest.raises(ValueError, match="global_dofs differs"):
        load_checkpoint(d, 5, compat(mpi_ranks=1, global_dofs=13))
    with pytest.raises(ValueError, match="does not match current finite-element space size"):
        load_checkpoint(d, 5, c, shape=(11,))
    # cycle mismatch and missing time in the metadata
    md = json.load(open(cfg.metadata_file(5)))
    json.dump(dict(md, cycle=9), open(cfg.metadata_file(5), "w"))
    with pytest.raises(ValueError, match="cycle mismatch: requested 5 but metadata contains 9"):
        load_checkpoint(d, 5, c)
    json.dump({k: v for k, v in md.items() if k != "time"}, open(cfg.metadata_file(5), "w"))
    with pytest.raises(ValueError, match="simulation time"):
        load_checkpoint(d, 5, c)
    # legacy metadata names an MFEM grid-function state, not read here
    json.dump({"time": 1.5, "cycle": 5}, open(cfg.metadata_file(5), "w"))
    with pytest.raises(NotImplementedError, match="Legacy"):
        load_checkpoint(d, 5, c)
    # a damaged header
    json.dump(md, open(cfg.metadata_file(5), "w"))
    raw = open(cfg.rank_file(5, 0), "rb").read()
    open(cfg.rank_file(5, 0), "wb").write(b"X" + raw[1:])
    with pytest.raises(ValueError, match="Invalid checkpoint state header"):
        load_checkpoint(d, 5, c)


def test_reads_a_state_written_by_a_plain_writer(tmp_path):
    """A checkpoint produced outside the library (as the reference writes it)
    loads unchanged."""
    d = tmp_path / "Checkpoints" / "Cycle3"
    d.mkdir(parents=True)
    u = np.linspace(-1.0, 1.0, 24)
    with open(d / "checkpoint_cycle_3.00000000.chk", "wb") as f:
        f.write(b"THESEUS_CHECKPOINT_RAW_V1\n" + struct.pack("<Q", u.size) + u.astype("<f8").tobytes())
    md = {"format_version": 2, "state_format": "raw_vector_v1", "state_representation": "conservative",
          "geometry": "cartesian", "real_bytes": 8, "time": 0.75, "cycle": 3, "mpi_ranks": 1,
          "order": 2, "dimension": 2, "num_equations": 4, "global_elements": 2, "global_dofs": 24}
    (d / "checkpoint_cycle_3.json").write_text(json.dumps(md, indent=2))
    c = CheckpointCompatibility(1, 2, 2, 4, 8, 2, 24)
    t, s = load_checkpoint(str(tmp_path / "Checkpoints"), 3, c)
    assert t == 0.75 and np.array_equal(s, u)
