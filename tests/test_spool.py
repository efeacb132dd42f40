"""RadioTrackSpool version 1 without a GPU: the reference's production
contract (testRadioTrackSpool.cpp:77-170: round trip in bounded batches,
rejected writes, empty and incomplete spools, six malformed files), the
byte layout read back independently, and make_host_radio_record
(HostRadioRecord.inl:11-31)."""
import math
import shutil
import struct

import numpy as np
import pytest


def track(pkg, index):
    """testRadioTrackSpool.cpp:47-61."""
    t = np.zeros((), pkg.abi.TRACK_SEGMENT)
    t["pdg"] = -11 if index % 2 else 11
    t["weight"] = 0.5 + index
    t["start_time_s"] = index * 1.e-7
    t["end_time_s"] = t["start_time_s"] + 3.e-9
    t["start_kinetic_energy_gev"] = 1.25
    t["end_kinetic_energy_gev"] = 1.2
    for axis in range(3):
        t["start_position_m"][axis] = axis + index * 0.25
        t["end_position_m"][axis] = t["start_position_m"][axis] + 0.5
        t["start_direction"][axis] = 1. if axis == 2 else 0.
        t["end_direction"][axis] = t["start_direction"][axis]
    return t


def tracks(pkg, count):
    return np.array([track(pkg, i) for i in range(count)], dtype=pkg.abi.TRACK_SEGMENT)


def test_production_contract(pkg, tmp_path):
    valid = tmp_path / "tracks.bin"
    writer = pkg.SpoolWriter(valid)
    writer.append(tracks(pkg, 103))
    assert writer.count() == 103
    writer.complete()
    with pytest.raises(pkg.RadioError):
        writer.complete()
    with pytest.raises(pkg.RadioError):
        writer.append(tracks(pkg, 2)[1:])
    writer.close()
    with pytest.raises(pkg.RadioError):
        pkg.SpoolWriter(valid)

    reader = pkg.SpoolReader(valid)
    assert reader.count == 103 and reader.state() == (0, False)
    for bad in (0, 65537):
        with pytest.raises(pkg.RadioError):
            reader.read_batch(bad)
    got = []
    while True:
        batch = reader.read_batch(7)
        if batch.size == 0:
            break
        assert batch.size <= 7
        got.append(batch)
    got = np.concatenate(got)
    want = tracks(pkg, 103)
    for field in want.dtype.names:
        assert np.array_equal(got[field], want[field]), field
    assert reader.state() == (103, True)
    reader.close()

    empty = tmp_path / "empty.bin"
    writer = pkg.SpoolWriter(empty)
    for field, value in (("pdg", 13), ("weight", -1.), ("end_time_s", -1.)):
        bad = track(pkg, 1)
        bad[field] = value
        with pytest.raises(pkg.RadioError):
            writer.append(np.array([bad]))
    bad = track(pkg, 1)
    bad["start_position_m"][1] = math.nan
    with pytest.raises(pkg.RadioError):
        writer.append(np.array([bad]))
    writer.complete()
    writer.close()
    reader = pkg.SpoolReader(empty)
    assert reader.count == 0 and reader.state() == (0, True) and reader.read_batch().size == 0
    reader.close()

    incomplete = tmp_path / "incomplete.bin"
    writer = pkg.SpoolWriter(incomplete)
    writer.append(tracks(pkg, 2)[1:])
    writer.close()  # destroyed without completion: the count stays all ones
    with pytest.raises(pkg.RadioError):
        pkg.SpoolReader(incomplete)

    for name, offset in (("bad-magic", 0), ("bad-version", 16), ("bad-size", 20), ("short", None),
                         ("extra", None), ("bad-value", 36)):
        malformed = tmp_path / name
        shutil.copy(valid, malformed)
        data = bytearray(malformed.read_bytes())
        if name == "short":
            data = data[:-1]
        elif name == "extra":
            data += b"\0"
        elif name == "bad-value":
            data[offset:offset + 8] = struct.pack("<d", math.nan)
        else:
            data[offset] = ord("!")
        malformed.write_bytes(bytes(data))
        with pytest.raises(pkg.RadioError):
            r = pkg.SpoolReader(malformed)
            r.read_batch(4096)


def test_byte_layout(pkg, tmp_path):
    path = tmp_path / "layout.bin"
    writer = pkg.SpoolWriter(path)
    writer.append(tracks(pkg, 2))
    writer.complete()
    writer.close()
    data = path.read_bytes()
    assert len(data) == 32 + 2 * 140
    assert data[:16] == b"C8_RADIO_TRACKS\0"
    assert struct.unpack("<IIQ", data[16:32]) == (1, 140, 2)
    for i in range(2):
        record = data[32 + 140 * i: 32 + 140 * (i + 1)]
        pdg = struct.unpack("<I", record[:4])[0]
        values = struct.unpack("<17d", record[4:])
        t = track(pkg, i)
        assert pdg == (11 if i % 2 == 0 else (1 << 32) - 11)
        want = (list(t["start_position_m"]) + list(t["end_position_m"]) + list(t["start_direction"]) +
                list(t["end_direction"]) + [t["start_time_s"], t["end_time_s"], t["start_kinetic_energy_gev"],
                                            t["end_kinetic_energy_gev"], t["weight"]])
        assert list(values) == [float(v) for v in want]


def test_host_record_conversion(pkg):
    seg = tracks(pkg, 3)
    records = pkg.track_records(seg)
    mass = 5.109989e-4
    assert np.array_equal(records["start"]["pid"], seg["pdg"])
    assert np.array_equal(records["end"]["pid"], seg["pdg"])
    assert np.array_equal(records["start"]["energy_gev"], seg["start_kinetic_energy_gev"] + mass)
    assert np.array_equal(records["end"]["energy_gev"], seg["end_kinetic_energy_gev"] + mass)
    assert np.array_equal(records["start"]["position_m"], seg["start_position_m"])
    assert np.array_equal(records["end"]["direction"], seg["end_direction"])
    assert np.array_equal(records["start"]["time_s"], seg["start_time_s"])
    assert np.array_equal(records["end"]["weight"], seg["weight"])
    bad = seg.copy()
    bad["pdg"][1] = 22
    with pytest.raises(pkg.InvalidArgument):
        pkg.track_records(bad)
