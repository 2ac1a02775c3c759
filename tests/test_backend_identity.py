"""The checkpoint's backend identity of a run on this library, mirrored from
the reference's checkpoint and provenance code (my-version/src/
checkpoint.rs:89-160, :1133-1175, provenance.rs:13-121, main.rs:4174-4206):
the records, the resume refusal and its exact message, the allowed-change
note and the build-identity differences. Runs on the CPU."""
import pytest


def test_records_and_error_kind(pkg):
    h = pkg.host
    assert h.checkpoint_backend_records() == ["backend gpu", "error_kind f32_proxy"]
    assert [h.error_kind_for_backend(b) for b in h.BACKENDS] == ["f64", "f32_proxy", "unknown"]
    with pytest.raises(ValueError) as e:
        h.parse_backend("tpu")
    assert str(e.value) == "backend must be 'cpu', 'gpu' or 'unknown', got 'tpu'"
    ident = h.BuildIdentity("0.1.0", "abc", "ff", "NVIDIA B200 (sm_100, 148 SMs, 183359 MB)",
                            "580.159", 16)
    recs = h.checkpoint_backend_records(ident)
    assert recs[2:] == ["build version 0.1.0", "build commit abc", "build binary_sha256 ff",
                        "build device NVIDIA B200 (sm_100, 148 SMs, 183359 MB)",
                        "build driver 580.159", "build threads 16"]


def test_resume_across_backends(pkg):
    h = pkg.host
    with pytest.raises(h.CheckpointMismatch) as e:
        h.check_backend("gpu", "cpu")
    assert str(e.value) == (
        "checkpoint backend mismatch: saved run used 'gpu', this run uses 'cpu'; pass "
        "--allow-backend-change to resume across backends (the trajectory and reported "
        "errors will differ)")
    h.check_backend("gpu", "cpu", allow_change=True)
    assert h.backend_change_note("gpu", "cpu") == (
        "# checkpoint: backend changed gpu -> cpu (allowed by --allow-backend-change)")
    # same backend, or a checkpoint from before the record: nothing to check or say
    h.check_backend("gpu", "gpu")
    h.check_backend("unknown", "gpu")
    assert h.backend_change_note("gpu", "gpu") is None
    assert h.backend_change_note("unknown", "cpu") is None


def test_build_identity_differences(pkg):
    """provenance.rs:101-121: each changed field is named in order; device
    and driver are ignored across a backend change."""
    h = pkg.host
    a = h.BuildIdentity("0.1.0", "abc", "ff", "cpu", "n/a", 8)
    assert a.differences(a) == []
    b = h.BuildIdentity("0.1.0", "deadbeef", "ff", "cpu", "n/a", 9)
    d = a.differences(b)
    assert len(d) == 2 and d[0].startswith("commit: ") and d[1].startswith("threads: ")
    gpu = h.BuildIdentity("0.1.0", "abc", "ff", "NVIDIA", "1", 8)
    assert a.differences(gpu) == []
    other = h.BuildIdentity("0.1.0", "abc", "ff", "NVIDIA H100", "2", 8)
    assert gpu.differences(other) == ["device: saved NVIDIA -> current NVIDIA H100",
                                      "driver: saved 1 -> current 2"]
    with pytest.raises(h.CheckpointMismatch) as e:
        h.check_identity(gpu, other)
    assert str(e.value).startswith("checkpoint build identity mismatch (device: saved NVIDIA")
    h.check_identity(gpu, other, allow_change=True)
    h.check_identity(None, other)
    assert h.device_identity(False) == ("cpu", "n/a")


@pytest.mark.gpu
def test_gpu_identity_names_the_device(pkg):
    """On a B200 the identity's device is the library's rc_device_name."""
    device, driver = pkg.host.device_identity(True)
    assert "B200" in device and "sm_100" in device, device
    assert driver != "n/a"
