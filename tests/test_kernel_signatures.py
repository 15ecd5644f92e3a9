"""CPU-only source check of the CUDA kernels' parameter lists.

A kernel that receives a large struct by plain value and passes its address on (here: the
potential descriptor handed by reference to the out-of-line pot_eval) makes every thread copy the
whole struct into local memory first.  Marked `const __grid_constant__`, the parameter is read in
place.  The job-set-up kernels once paid more than half their time for that copy, so every
`__global__` parameter whose type is, or embeds, the potential descriptor must carry the qualifier.
"""
import os
import re

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "zinq_b200", "csrc")

# PotDev, and the structs that hold one by value (LineJob reaches kernels only through pointers)
EMBEDS_POTENTIAL = ("PotDev", "NdJob", "LineTablesArgs", "GapArgs", "LineJob")


def kernel_signatures():
    """(file, kernel name, [parameter declarations]) of every __global__ function in csrc."""
    out = []
    for name in sorted(os.listdir(CSRC)):
        if not name.endswith((".cu", ".cuh")):
            continue
        text = open(os.path.join(CSRC, name)).read()
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"__global__", text):
            pos = m.end()
            while True:  # the first `name(` after __global__ that is not __launch_bounds__(...)
                head = re.compile(r"(\w+)\s*\(").search(text, pos)
                start = head.end()
                depth, i = 1, start
                while depth:
                    depth += {"(": 1, ")": -1}.get(text[i], 0)
                    i += 1
                if head.group(1) != "__launch_bounds__":
                    break
                pos = i
            params = [p.strip() for p in text[start:i - 1].split(",") if p.strip()]
            out.append((name, head.group(1), params))
    return out


def test_signatures_are_found():
    names = {k for _, k, _ in kernel_signatures()}
    for k in ("nd_table_kernel", "line_tables_kernel", "min_gap_kernel", "potential_plot_kernel",
              "nd_row_tma_kernel", "nd_tile_tma_kernel", "line_solve_kernel"):
        assert k in names, k


def test_potential_structs_are_grid_constant():
    bad = []
    for fname, kernel, params in kernel_signatures():
        for p in params:
            tokens = re.findall(r"\w+|[*&]", p)
            if not any(t in EMBEDS_POTENTIAL for t in tokens) or "*" in tokens or "&" in tokens:
                continue
            if "__grid_constant__" not in tokens or "const" not in tokens:
                bad.append(f"{fname}: {kernel}({p})")
    assert not bad, "by-value struct parameters without const __grid_constant__:\n" + "\n".join(bad)
