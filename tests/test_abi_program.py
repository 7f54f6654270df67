"""A plain-C99 host program (tests/abi/frame_loop.c) drives the reference
app's frame loop through the C ABI alone: the manager from a treelet file,
the device buffer, analysis passes with paging, a frame into host memory.
The header must compile as strict C and the program must link against the
library (CPU); on a GPU its last frame must equal the oracle's over the pool
it ended with, and that pool the one the Python mirror reaches with the same
steps."""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import libsvo_b200 as L

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
SRC = HERE / "abi" / "frame_loop.c"
EXE = HERE / "abi" / "_build" / "frame_loop"
SRC_CPP = HERE / "abi" / "frame_loop.cpp"
EXE_CPP = HERE / "abi" / "_build" / "frame_loop_cpp"


def build_program() -> Path:
    lib_dir = Path(L.LIB_PATH).parent
    EXE.parent.mkdir(parents=True, exist_ok=True)
    subprocess.run(["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    f"-I{ROOT / 'include'}", str(SRC), "-o", str(EXE), f"-L{lib_dir}", "-lsvo_b200",
                    f"-Wl,-rpath,{lib_dir}"], check=True, capture_output=True, text=True)
    return EXE


def build_cpp_program() -> Path:
    """tests/abi/frame_loop.cpp against the header-only C++ class
    (include/libsvo_b200.hpp)."""
    lib_dir = Path(L.LIB_PATH).parent
    EXE_CPP.parent.mkdir(parents=True, exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    f"-I{ROOT / 'include'}", str(SRC_CPP), "-o", str(EXE_CPP), f"-L{lib_dir}", "-lsvo_b200",
                    f"-Wl,-rpath,{lib_dir}"], check=True, capture_output=True, text=True)
    return EXE_CPP


def test_header_is_c99_and_the_program_links():
    exe = build_program()
    assert exe.is_file() and os.access(exe, os.X_OK)


def test_cpp_class_header_compiles_and_links():
    exe = build_cpp_program()
    assert exe.is_file() and os.access(exe, os.X_OK)


@pytest.mark.gpu
def test_c_frame_loop_matches_oracle_and_python(cuda, tmp_path):
    import oracle

    exe = build_program()
    scene = L.Scene.menger(level=4, depth=7, seed=9, treelet_levels=3)
    base = tmp_path / "menger"
    scene.write(str(base))
    info = scene.info
    incore = info.treelet_bytes * max(2, info.num_treelets * 2 // 3)  # paging with eviction
    frames = [L.orbit_camera(30 + i, 160, 120, radius=(1.2, 1.9)).frame_params(t_scale_ratio=0.0)
              for i in range(6)]
    params = tmp_path / "params.bin"
    params.write_bytes(b"".join(bytes(p) for p in frames))
    out = tmp_path / "out"
    r = subprocess.run([str(exe), str(base), str(incore), str(len(frames)), str(params), str(out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("placed ")
    last = frames[-1]
    rgba = np.fromfile(str(out) + ".rgba", dtype=np.uint32).reshape(last.height, last.width)
    nodes = np.fromfile(str(out) + ".nodes", dtype=np.uint32).reshape(-1, 2)
    attribs = np.fromfile(str(out) + ".attribs", dtype=np.uint32).reshape(-1, 2)
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(last))
    assert np.array_equal(rgba, o_rgba)
    assert o_hits["hit"].sum() > 500
    # the Python mirror through the same calls ends with the same pool
    mm = L.TreeletMemoryManagerCuda(str(base), incore)
    mm.initDeviceBuffer()
    for p in frames:
        mm.performAnalysePass(p, divisor=1)
    pn, pa = mm.getIncoreBuffer()
    assert np.array_equal(pn, nodes) and np.array_equal(pa, attribs)
    mm.close()


@pytest.mark.gpu
def test_cpp_class_frame_loop_matches_oracle_and_c_program(cuda, tmp_path):
    """The same frame loop through svo::TreeletMemoryManagerCuda (reference
    method names): its last frame equals the oracle's over its final pool, and
    that pool equals the C program's after the same steps."""
    import oracle

    exe_c, exe_cpp = build_program(), build_cpp_program()
    scene = L.Scene.menger(level=4, depth=7, seed=9, treelet_levels=3)
    base = tmp_path / "menger"
    scene.write(str(base))
    info = scene.info
    incore = info.treelet_bytes * max(2, info.num_treelets * 2 // 3)
    frames = [L.orbit_camera(40 + i, 128, 96, radius=(1.2, 1.9)).frame_params(t_scale_ratio=0.0)
              for i in range(5)]
    params = tmp_path / "params.bin"
    params.write_bytes(b"".join(bytes(p) for p in frames))
    outs = {}
    for name, exe in (("c", exe_c), ("cpp", exe_cpp)):
        out = tmp_path / name
        r = subprocess.run([str(exe), str(base), str(incore), str(len(frames)), str(params), str(out)],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (name, r.returncode, r.stderr)
        outs[name] = out
    last = frames[-1]
    rgba = np.fromfile(str(outs["cpp"]) + ".rgba", dtype=np.uint32).reshape(last.height, last.width)
    nodes = np.fromfile(str(outs["cpp"]) + ".nodes", dtype=np.uint32).reshape(-1, 2)
    attribs = np.fromfile(str(outs["cpp"]) + ".attribs", dtype=np.uint32).reshape(-1, 2)
    o_rgba, o_hits, _, _ = oracle.render(nodes, attribs, bytes(last))
    assert np.array_equal(rgba, o_rgba)
    assert o_hits["hit"].sum() > 300
    for ext in (".nodes", ".attribs"):
        assert np.array_equal(np.fromfile(str(outs["c"]) + ext, dtype=np.uint32),
                              np.fromfile(str(outs["cpp"]) + ext, dtype=np.uint32)), ext
