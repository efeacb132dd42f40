"""The output step on the device (RadioProcess.inl:213-223, the observer add of
CorsikaOutputSink.inl:255-278): decoded CoREAS fields and ZHS fields
-(A[i+1] - A[i]) fs added into device buffers equal the same computation on
the host from download(), bit for bit, also when two showers add up."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def host_fields(w, observers):
    """CoREAS as downloaded; ZHS differentiated per observer, as RadioProcess.inl:215-218."""
    zhs = []
    offset = 0
    fs = observers["sample_rate_hz"]
    for o, n in enumerate(observers["number_of_bins"]):
        a = w.zhs[:, offset:offset + int(n)]
        zhs.append(-(a[:, 1:] - a[:, :-1]) * fs[o])
        offset += int(n)
    return w.coreas, np.concatenate(zhs, axis=1)


@pytest.mark.parametrize("deterministic", [True, False])
def test_device_output_step_matches_host(pkg, showers, deterministic):
    import torch

    wl, gen, _ = showers.workload_config("plain_c0", bins=1024)
    observers = wl["observers"]
    config = showers.make_config(wl, precision=1, kernel=2, deterministic=deterministic)
    events = [showers.shower_records(15000, seed=s, **gen) for s in (71, 72)]
    nc = int(observers["number_of_bins"].sum())
    coreas = torch.zeros(3 * nc, dtype=torch.float64, device="cuda")
    zhs = torch.zeros(3 * (nc - observers.size), dtype=torch.float64, device="cuda")
    want = None
    for records in events:
        raw = torch.from_numpy(records.view(np.uint8).reshape(-1)).cuda()
        acc = pkg.RadioAccumulator(config)
        acc.accumulate_lepton_tracks(raw.data_ptr(), records.size)
        acc.download_fields_device(coreas.data_ptr(), zhs.data_ptr())
        acc.close()
        reference = pkg.RadioAccumulator(config)
        reference.accumulate_lepton_tracks(raw.data_ptr(), records.size)
        fields = host_fields(reference.download(), observers)
        reference.close()
        want = fields if want is None else (want[0] + fields[0], want[1] + fields[1])
    torch.cuda.synchronize()
    got = (coreas.cpu().numpy().reshape(3, -1), zhs.cpu().numpy().reshape(3, -1))
    if deterministic:
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    else:  # FP64 atomics: the two projections sum in different orders
        for g, w in zip(got, want):
            assert np.abs(g - w).max() <= 1e-12 * np.abs(w).max()
