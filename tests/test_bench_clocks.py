"""bench.py's clock sampler against a stand-in `nvidia-smi` on PATH (a shell loop printing the
queried CSV fields): samples land in the directory given, only those after mark() count, and the
summary carries the median SM clock, the maximum and the active throttle reasons."""
import os
import stat
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

FAKE = """#!/bin/sh
# index, clocks.sm, clocks.max.sm, power.draw, active, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
i=0
while [ $i -lt 400 ]; do
  if [ -f "$FAKE_SMI_PHASE" ]; then
    echo "0, 1965, 1965, 640.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active"
  else
    echo "0, 345, 1965, 95.0, 0x0000000000000001, Not Active, Not Active, Not Active, Not Active"
  fi
  i=$((i+1))
  sleep 0.01
done
"""


def test_clock_sampler_with_stand_in_nvidia_smi(tmp_path, monkeypatch):
    bindir = tmp_path / "bin"
    bindir.mkdir()
    smi = bindir / "nvidia-smi"
    smi.write_text(FAKE)
    smi.chmod(smi.stat().st_mode | stat.S_IEXEC)
    phase = tmp_path / "loaded"
    monkeypatch.setenv("PATH", f"{bindir}{os.pathsep}{os.environ['PATH']}")
    monkeypatch.setenv("FAKE_SMI_PHASE", str(phase))
    out = tmp_path / "clocks"
    c = bench.ClockSampler(0, str(out))
    c.start()
    c.wait_first_sample()
    time.sleep(0.1)  # idle samples before the timed region
    c.mark()
    phase.write_text("")
    time.sleep(0.5)
    info = c.stop()
    assert (out / "clocks_rank0.csv").exists()
    assert info is not None and info["samples"] >= 5
    # the few samples taken between mark() and the phase switch are idle ones; the median is loaded
    assert info["sm_mhz"] == 1965.0 and info["sm_max_mhz"] == 1965.0
    assert info["reasons"] == ["sw_power_cap"]


def test_clock_sampler_without_nvidia_smi(tmp_path, monkeypatch):
    monkeypatch.setenv("PATH", str(tmp_path))
    c = bench.ClockSampler(0, str(tmp_path / "clocks"))
    c.start()
    c.wait_first_sample(timeout=0.2)
    c.mark()
    assert c.stop() is None


def test_sampler_reads_the_gpu_behind_cuda_visible_devices(monkeypatch):
    """CUDA device k of the process is the k-th entry of CUDA_VISIBLE_DEVICES, which is what
    nvidia-smi --id must be given (an index or a UUID)."""
    monkeypatch.delenv("CUDA_VISIBLE_DEVICES", raising=False)
    assert bench.nvsmi_device(3) == "3"
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "5,2")
    assert bench.nvsmi_device(0) == "5" and bench.nvsmi_device(1) == "2"
    monkeypatch.setenv("CUDA_VISIBLE_DEVICES", "GPU-1234abcd")
    assert bench.nvsmi_device(0) == "GPU-1234abcd"
