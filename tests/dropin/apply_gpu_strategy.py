#!/usr/bin/env python3
"""Applies the integration patch (StorageStrategyKind::Gpu) to a copy of the
TMFQS source tree, in place.

    python tests/dropin/apply_gpu_strategy.py <copy-of-the-reference-tree>

The edits are the ones a maintainer makes to adopt the device backend; each
is anchored on the reference's own text and fails loudly when the anchor is
missing, so a changed reference is noticed instead of silently mis-patched:

1. include/tmfqs/config/register_config.h: a `Gpu` value at the end of
   StorageStrategyKind (after `Auto`).
2. src/tmfqs/storage/factory/storage_strategy_registry.cpp: Gpu in
   isAvailable, listAvailable ("gpu"), toString ("gpu") and createSelection
   (createGpuStateBackend, with the reference's "requested but unavailable"
   error); plus the test-harness switch: with TMFQS_DENSE_BACKEND=gpu in the
   environment, Dense registers are built on the device backend too.
3. examples/grover_cli.h and examples/qftG.cpp: `--strategy gpu`.
4. The backend itself: tests/dropin/gpu_state_backend.{h,cpp} into
   include/tmfqs/storage/gpu/ and src/tmfqs/storage/gpu/.
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def edit(path, old, new):
    with open(path) as f:
        s = f.read()
    if old not in s:
        raise SystemExit(f"anchor not found in {path}: {old!r}")
    with open(path, "w") as f:
        f.write(s.replace(old, new, 1))


def main(tree):
    cfg = os.path.join(tree, "include/tmfqs/config/register_config.h")
    edit(cfg, "\tAuto\n};", "\tAuto,\n\t/** @brief B200 device state vector (libtmfqs_b200). */\n\tGpu\n};")

    reg = os.path.join(tree, "src/tmfqs/storage/factory/storage_strategy_registry.cpp")
    edit(reg, '#include "tmfqs/storage/dense/dense_state_backend.h"\n',
         '#include "tmfqs/storage/dense/dense_state_backend.h"\n#include "tmfqs/storage/gpu/gpu_state_backend.h"\n')
    edit(reg, "\t\tcase StorageStrategyKind::Auto:\n\t\t\treturn true;\n",
         "\t\tcase StorageStrategyKind::Gpu:\n\t\t\treturn isGpuStateBackendAvailable();\n"
         "\t\tcase StorageStrategyKind::Auto:\n\t\t\treturn true;\n")
    edit(reg, '\tnames.push_back("auto");\n',
         '\tif(isGpuStateBackendAvailable()) {\n\t\tnames.push_back("gpu");\n\t}\n\tnames.push_back("auto");\n')
    edit(reg, '\t\tcase StorageStrategyKind::Auto:\n\t\t\treturn "auto";\n',
         '\t\tcase StorageStrategyKind::Gpu:\n\t\t\treturn "gpu";\n\t\tcase StorageStrategyKind::Auto:\n\t\t\treturn "auto";\n')
    edit(reg, "\t\t\tselection.backend = createDenseStateBackend(selection.config);\n",
         "\t\t\tselection.backend = denseRedirectedToGpu() ? createGpuStateBackend(selection.config)\n"
         "\t\t\t                                           : createDenseStateBackend(selection.config);\n")
    edit(reg, "\t\tcase StorageStrategyKind::Auto:\n\t\t\tthrow",
         "\t\tcase StorageStrategyKind::Gpu:\n\t\t\tselection.backend = createGpuStateBackend(selection.config);\n"
         "\t\t\tif(!selection.backend) {\n\t\t\t\tthrow std::runtime_error(\"Gpu backend requested but unavailable in this build\");\n"
         "\t\t\t}\n\t\t\tbreak;\n\t\tcase StorageStrategyKind::Auto:\n\t\t\tthrow")

    for ex in ("examples/grover_cli.h", "examples/qftG.cpp"):
        edit(os.path.join(tree, ex), '\tif(value == "auto") return tmfqs::StorageStrategyKind::Auto;\n',
             '\tif(value == "auto") return tmfqs::StorageStrategyKind::Auto;\n'
             '\tif(value == "gpu") return tmfqs::StorageStrategyKind::Gpu;\n')

    os.makedirs(os.path.join(tree, "include/tmfqs/storage/gpu"), exist_ok=True)
    os.makedirs(os.path.join(tree, "src/tmfqs/storage/gpu"), exist_ok=True)
    shutil.copy(os.path.join(HERE, "gpu_state_backend.h"), os.path.join(tree, "include/tmfqs/storage/gpu/gpu_state_backend.h"))
    shutil.copy(os.path.join(HERE, "gpu_state_backend.cpp"), os.path.join(tree, "src/tmfqs/storage/gpu/gpu_state_backend.cpp"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    main(sys.argv[1])
