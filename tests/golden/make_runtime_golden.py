"""Regenerates tests/golden/runtime/ from upstream's own container code.

Requires oracle/_ref/libontc_ref_rt.so (`make -C oracle ref`, which compiles upstream's
libopenntc/openntc_runtime.cpp).  Writes:
  * case_<seed>.ntc      -- upstream Dump() of tests/golden/cases.Case(seed)
  * load_results.json    -- upstream Load() result codes for the malformed variants of case 0

Run from the repository root:  python tests/golden/make_runtime_golden.py
"""
import ctypes as C
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from oracle.bindings import RefRuntime  # noqa: E402
from tests.golden.cases import Case, corruptions  # noqa: E402

SEEDS = list(range(12))


def main():
    ref = RefRuntime()
    out = HERE / "runtime"
    out.mkdir(exist_ok=True)
    for s in SEEDS:
        c = Case(s)
        p = out / f"case_{s}.ntc"
        assert ref.L.ref_rt_dump(str(p).encode(), C.byref(c.data)) == 0
    raw = (out / "case_0.ntc").read_bytes()
    results = {}
    tmp = out / "_tmp.ntc"
    for name, blob in corruptions(raw).items():
        tmp.write_bytes(blob)
        h = C.c_void_p()
        cd = (C.c_uint8 * ref.L.ref_rt_sizeof_compressed())()
        r = ref.L.ref_rt_load(str(tmp).encode(), C.byref(h), cd)
        ref.L.ref_rt_free(h)
        results[name] = r
    tmp.unlink()
    (out / "load_results.json").write_text(json.dumps(results, indent=1, sort_keys=True))
    print("wrote", len(SEEDS), "containers and", len(results), "load results")


if __name__ == "__main__":
    main()
