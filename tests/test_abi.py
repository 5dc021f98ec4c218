"""The C ABI: libcpx.so loads, exports every function include/cpx.h declares, and
rejects invalid arguments before touching the device (no GPU needed)."""
import ctypes as C
import re

import pytest

from conftest import REPO


def header_functions():
    text = (REPO / "include" / "cpx.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cpx_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_reference_entry_points():
    names = header_functions()
    for must in ("cpx_render_forward", "cpx_render_backward", "cpx_tv_grad", "cpx_adam_step",
                 "cpx_grid_create", "cpx_grid_upload_params", "cpx_occupancy_build", "cpx_rays_init_camera"):
        assert must in names


def test_library_exports_every_declared_symbol():
    import cpx

    lib = C.CDLL(str(cpx.LIB_PATH))
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, f"libcpx.so lacks {missing}"
    assert sorted(cpx.EXPORTED) == header_functions()


def test_status_strings_and_version():
    import cpx

    assert cpx.version() >= 100
    assert cpx._lib.cpx_status_string(0) == b"ok"
    assert cpx._lib.cpx_status_string(4).startswith(b"march")


@pytest.mark.parametrize("kw,status", [
    (dict(width=1, height=8, depth=8), "CPX_ERR_INVALID_ARGUMENT"),
    (dict(sh_dim=5), "CPX_ERR_UNSUPPORTED"),
    (dict(sh_dim=4, optimizing_band=2), "CPX_ERR_INVALID_ARGUMENT"),
    (dict(step_size=0.0), "CPX_ERR_INVALID_ARGUMENT"),
    (dict(step_size=float("nan")), "CPX_ERR_INVALID_ARGUMENT"),
    (dict(width=2048, height=2048, depth=1024), "CPX_ERR_INVALID_ARGUMENT"),
])
def test_grid_create_rejects_invalid_descriptions(kw, status):
    import cpx

    args = dict(width=8, height=8, depth=8, sh_dim=9, step_size=0.5)
    args.update(kw)
    band = args.pop("optimizing_band", None)
    with pytest.raises(cpx.CpxError) as ei:
        cpx.ObjectScene(args.pop("width"), args.pop("height"), args.pop("depth"), optimizing_band=band, **args)
    assert ei.value.name == status


def test_null_handles_are_rejected():
    import cpx

    assert cpx._lib.cpx_grid_check(None) == 1
    assert cpx._lib.cpx_tv_grad(None, 0.0, 0.0, 0, 6, None) == 1
    assert cpx._lib.cpx_rays_create(-1, 1, C.byref(C.c_void_p())) == 1


def test_oracle_library_loads():
    import orc

    assert orc.threads() >= 1
