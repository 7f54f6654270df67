"""The library's host code under AddressSanitizer and UndefinedBehavior-
Sanitizer: the library rebuilt with instrumented host objects
(libsvo_b200/_build.py build_sanitized) runs the host-side test modules -- the
memory manager's slot bookkeeping and patching, the analysis, the scene
builder and treelet files, PLY input, the C ABI's argument checks -- in a
child process with the sanitizer runtimes preloaded.  Any invalid access,
use after free or undefined behaviour aborts the child."""
import os
import subprocess
import sys
from pathlib import Path

import __graft_entry__

ROOT = Path(__file__).resolve().parent.parent
HOST_MODULES = ["test_memory_manager.py", "test_analysis.py", "test_scene.py", "test_mesh_io.py",
                "test_capi.py"]


def test_host_code_under_asan_and_ubsan():
    b = __graft_entry__._load_build_module()
    lib = b.build_sanitized()
    env = dict(os.environ)
    env.update({"LD_PRELOAD": b.sanitizer_preload(), "LIBSVO_B200_LIB": str(lib),
                "ASAN_OPTIONS": "detect_leaks=0:protect_shadow_gap=0:abort_on_error=1",
                "UBSAN_OPTIONS": "halt_on_error=1:print_stacktrace=1"})
    r = subprocess.run([sys.executable, "-m", "pytest", "-x", "-q", "-m", "not gpu", "-p", "no:cacheprovider",
                        *[str(ROOT / "tests" / m) for m in HOST_MODULES]],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    tail = (r.stdout + r.stderr)[-3000:]
    assert r.returncode == 0, tail
    assert "passed" in r.stdout and "AddressSanitizer" not in r.stderr and "runtime error" not in r.stderr, tail
