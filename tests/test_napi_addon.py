"""The Node.js N-API addon (kraken_3_gpu_b200/napi) that binds the drop-in
C ABI for the reference's JavaScript: it compiles (gcc, -Werror, against the
Node-API declarations), exports the module entry point Node looks up, calls
only Node-API functions and this library's declared C entry points, and its
JS module exports the gpuworld.js surface (src/gpu/gpuworld.js:28-472)."""
import os
import re
import subprocess

from kraken_3_gpu_b200 import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NAPI = os.path.join(ROOT, "kraken_3_gpu_b200", "napi")


def _syms(obj, flag):
    out = subprocess.run(["nm", flag, obj], check=True, capture_output=True, text=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


def test_addon_compiles_and_exports_the_module_entry_point():
    obj = build.build_napi_object()
    assert _syms(obj, "--defined-only") & {"napi_register_module_v1"} == {"napi_register_module_v1"}
    exported = {s for s in _syms(obj, "-g") if not s.startswith(("napi_", "kr_", "__", "calloc", "free"))}
    undefined = _syms(obj, "-u")
    napi = {s for s in undefined if s.startswith("napi_")}
    declared = set(re.findall(r"\b(napi_[a-z0-9_]+)\s*\(", open(os.path.join(NAPI, "node_api_decls.h")).read()))
    assert napi and napi <= declared
    kr = {s for s in undefined if s.startswith("kr_")}
    header = open(os.path.join(ROOT, "include", "kraken_b200.h")).read()
    for s in kr:
        assert re.search(rf"\b{s}\s*\(", header), f"{s} is not in include/kraken_b200.h"
    assert {"kr_create", "kr_upload", "kr_upload_controls", "kr_step", "kr_download", "kr_destroy"} <= kr
    assert exported == set(), exported


def test_js_module_exports_the_gpuworld_surface():
    src = open(os.path.join(NAPI, "gpuworld_cuda.js")).read()
    names = set(re.findall(r"export (?:async )?function (\w+)", src))
    names |= {n.strip() for m in re.findall(r"export \{([^}]*)\}", src) for n in m.split(",")}
    want = {"GPU_STRIDES", "isAvailable", "create", "groupCollPoints", "upload", "uploadControls",
            "packControls", "step", "download", "mirrorInto", "destroy", "loadWgsl"}
    assert want <= names, want - names
    addon_calls = set(re.findall(r"addon\.(\w+)\(", src))
    c = open(os.path.join(NAPI, "kraken_napi.c")).read()
    registered = set(re.findall(r'export_fn\(env, exports, "(\w+)"', c))
    assert addon_calls <= registered, addon_calls - registered
