"""The branch-free forms of the star path against the forms they replace,
bit for bit, on the host (tests/cpp/star_forms.cu, compiled by nvcc as host
code: no GPU): the quad test from the pixel's edge terms against in_quad
(starInPolygon, BT/kernel.cuh:245-266) and the bisection with its quadrant
cases as selects against the cases as branches (interpolate,
BT/kernel.cuh:112-200)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "star_forms.cu")
EXE = os.path.join(ROOT, "tests", "cpp", "star_forms")
HDR = os.path.join(ROOT, "blacktracer_b200", "csrc", "stars_pixel.cuh")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def test_branch_free_star_forms_are_exact():
    deps = [SRC, HDR]
    if not os.path.exists(EXE) or os.path.getmtime(EXE) < max(os.path.getmtime(d) for d in deps):
        subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
                        "-I" + os.path.join(ROOT, "include"),
                        "-I" + os.path.join(ROOT, "blacktracer_b200", "csrc"), SRC, "-o", EXE],
                       check=True)
    out = subprocess.run([EXE], check=True, capture_output=True, text=True).stdout.split("\n")
    q_bad, q_n = (int(x) for x in out[0].split()[1:])
    b_bad, b_n = (int(x) for x in out[1].split()[1:])
    assert q_n >= 100_000 and b_n >= 50_000
    assert q_bad == 0, f"{q_bad} of {q_n} quad tests differ"
    assert b_bad == 0, f"{b_bad} of {b_n} bisections differ"
