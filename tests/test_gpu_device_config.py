"""Device configuration at vklCommitDevice, as the reference's
Device::commit (openvkl/api/Device.cpp:135-199) does it: errors go to stderr
as "OPENVKL ERROR [<code>]: <message>" by default; the errorOutput /
logOutput / logLevel parameters redirect or silence them, and the
OPENVKL_ERROR_OUTPUT / OPENVKL_LOG_OUTPUT / OPENVKL_LOG_LEVEL environment
variables take precedence over the parameters.  Each case runs in a child
process whose output is checked."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import ctypes as C, sys
sys.path.insert(0, %r)
from openvkl_b200 import vkl
L = vkl.load_library()
L.vklInit()
d = L.vklNewDevice(b"cuda")
assert d
for kv in sys.argv[1:]:
    k, v = kv.split("=")
    if k == "logLevel":
        L.vklDeviceSetInt(d, b"logLevel", int(v))
    else:
        L.vklDeviceSetString(d, k.encode(), v.encode())
L.vklCommitDevice(d)
L.vklNewVolume(d, b"no_such_volume_type")
print("code", L.vklDeviceGetLastErrorCode(d), flush=True)
""" % ROOT


def _run(args=(), env=None):
    e = dict(os.environ)
    for k in ("OPENVKL_ERROR_OUTPUT", "OPENVKL_LOG_OUTPUT", "OPENVKL_LOG_LEVEL"):
        e.pop(k, None)
    e.update(env or {})
    r = subprocess.run([sys.executable, "-c", SCRIPT, *args], capture_output=True, text=True, env=e, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout, r.stderr


def test_default_error_output_is_stderr(vkl):
    out, err = _run()
    assert "OPENVKL ERROR [2]: unsupported volume type 'no_such_volume_type'" in err
    assert "OPENVKL ERROR" not in out
    assert "code 2" in out


def test_error_output_parameter_and_environment(vkl):
    out, err = _run(["errorOutput=cout"])
    assert "OPENVKL ERROR [2]" in out and "OPENVKL ERROR" not in err
    out, err = _run(["errorOutput=none"])
    assert "OPENVKL ERROR" not in out + err and "code 2" in out
    # the environment variable wins over the parameter
    out, err = _run(["errorOutput=none"], env={"OPENVKL_ERROR_OUTPUT": "cerr"})
    assert "OPENVKL ERROR [2]" in err


def test_log_level_environment(vkl):
    out, err = _run(env={"OPENVKL_LOG_LEVEL": "bogus"})
    assert "unknown OPENVKL_LOG_LEVEL env value" in out
    # values are case-insensitive
    out, err = _run(env={"OPENVKL_LOG_LEVEL": "NONE"})
    assert "unknown OPENVKL_LOG_LEVEL" not in out + err
