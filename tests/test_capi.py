"""The C-ABI library loads and exports every entry point the public header declares.
No compute calls: this runs without a GPU."""
import ctypes as C

from mguso import _lib


def test_header_declares_entry_points():
    syms = _lib.header_symbols()
    assert "mguso_linear_solve" in syms and "mguso_bsr_spmv" in syms
    assert len(syms) >= 20


def test_library_exports_every_header_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [s for s in _lib.header_symbols() if not hasattr(lib, s)]
    assert not missing, f"declared in include/mguso_cuda.h but not exported: {missing}"


def test_header_is_plain_c_and_cpp():
    """The boundary header compiles as strict C99 and as C++17 on its own and includes only
    the standard C headers: plain pointers, sizes and opaque handles, no CUDA or torch types
    in the signatures."""
    import os
    import shutil
    import subprocess

    import pytest

    hdr = os.path.join(os.path.dirname(_lib.LIB_PATH), "..", "..", "include", "mguso_cuda.h")
    for cc, args in (("gcc", ["-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-x", "c"]),
                     ("g++", ["-std=c++17", "-Wall", "-Werror", "-x", "c++"])):
        if shutil.which(cc) is None:
            pytest.skip(f"{cc} not found")
        subprocess.run([cc, *args, "-fsyntax-only", hdr], check=True)
    includes = [ln.split()[1] for ln in open(hdr) if ln.startswith("#include")]
    assert set(includes) <= {"<stddef.h>", "<stdint.h>"}, includes


def test_version_and_last_error_without_gpu():
    lib = _lib.load()
    assert lib.mguso_version() >= 100
    buf = C.create_string_buffer(64)
    lib.mguso_last_error(buf, 64)  # empty on a fresh thread; must not crash


def test_invalid_arguments_are_rejected_without_gpu():
    lib = _lib.load()
    assert lib.mguso_linear_solver_create(None, 1, 32, 1, None) == 1  # INVALID_ARG
    assert "null" in _lib.last_error()


def _triangle_scene(**stitch):
    import numpy as np

    from mguso import scenes

    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    st = dict(index=[0, 0, 0, 1, 1, 1], weight=[1.0, 0.0, 0.0, 1.0, 0.0, 0.0], stiffness=1.0, l0=0.001, l_cap=0.01)
    st.update(stitch)
    return dict(positions=pos, velocities=np.zeros_like(pos), inv_mass=np.ones(3, np.float32),
                tris=np.array([[0, 1, 2]], np.uint32), shell_faces=np.zeros((0, 3), np.uint32), static_mask=None,
                stitch_idx=np.array([st["index"]], np.uint32), stitch_w=np.array([st["weight"]], np.float32),
                stitch_kl=np.array([[st["stiffness"], st["l0"], st["l_cap"]]], np.float32),
                colliders=np.zeros((0, 8), np.float32), params=scenes.default_params())


def test_scene_validation_rejects_nonsense_stitches_without_gpu():  # implicit.rs:3494-3535
    import math

    import numpy as np
    import pytest

    from mguso import MgusoError
    from mguso.solver import validate_scene

    validate_scene(_triangle_scene())
    bad = [dict(index=[0, 0, 0, 9, 9, 9]), dict(stiffness=-1.0), dict(l0=0.0), dict(l_cap=0.0005),
           dict(weight=[0.5, 0, 0, 1.0, 0, 0]), dict(weight=[1.0, 0, 0, 0.5, 0, 0]), dict(l0=math.nan)]
    for b in bad:
        with pytest.raises(MgusoError) as e:
            validate_scene(_triangle_scene(**b))
        assert e.value.code == 1 and "stitch" in str(e.value), b
    sc = _triangle_scene()
    sc["tris"] = np.array([[0, 1, 7]], np.uint32)
    with pytest.raises(MgusoError, match="triangle index"):
        validate_scene(sc)
    sc = _triangle_scene()
    sc["params"] = dict(sc["params"], dt=0.0)
    with pytest.raises(MgusoError, match="dt"):
        validate_scene(sc)
