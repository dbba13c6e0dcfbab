"""Place the reference's unmodified Python package in baseline/_ref, for the drop-in tests.

    python baseline/install_reference.py --reference <path of the zcmir checkout>
    (or set ZCMIR_REFERENCE)

The reference's own install (``pip install <checkout>``) runs its build backend
(scripts/build_backend.py), which downloads Zig and wgpu-native and compiles the WebGPU engine:
with no network (and no graphics stack to run that engine) it cannot complete. The Python
package itself (python/zcmir/, numpy only) needs no build, so this recipe copies its files
byte for byte to baseline/_ref/zcmir/ and writes their SHA-256 to baseline/_ref/MANIFEST. With
``ZCMIR_LIB`` naming this repository's libzcmir.so (and ``ZCMIR_WGPU`` any existing file: the
package insists on one, and zc_create ignores it), that package runs on the B200 engine
unchanged. baseline/_ref is not committed; it travels with the working tree to the GPU machine.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
from pathlib import Path

HERE = Path(__file__).resolve().parent
DEST = HERE / "_ref"


def install(ref) -> Path:
    src = Path(ref) / "python" / "zcmir"
    if not (src / "__init__.py").exists():
        raise SystemExit(f"{src} holds no zcmir package")
    pkg = DEST / "zcmir"
    if pkg.exists():
        shutil.rmtree(pkg)
    pkg.mkdir(parents=True)
    lines = []
    for f in sorted(src.glob("*.py")):
        shutil.copyfile(f, pkg / f.name)
        lines.append(f"{hashlib.sha256(f.read_bytes()).hexdigest()}  zcmir/{f.name}")
    (DEST / "MANIFEST").write_text("\n".join(lines) + "\n")
    return pkg


def verify() -> bool:
    """Every file listed in MANIFEST is present with its recorded hash."""
    man = DEST / "MANIFEST"
    if not man.exists():
        return False
    for line in man.read_text().splitlines():
        digest, name = line.split("  ", 1)
        f = DEST / name
        if not f.exists() or hashlib.sha256(f.read_bytes()).hexdigest() != digest:
            return False
    return True


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=os.environ.get("ZCMIR_REFERENCE"),
                    help="the zcmir checkout (default: $ZCMIR_REFERENCE)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference or set ZCMIR_REFERENCE")
    print(install(a.reference))
