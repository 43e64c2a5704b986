"""The correctly rounded exp of yuzen_b200/csrc/yz_exp.h: on the CPU (the
header compiled by g++, as the ConcZ oracle links it in place of the libm's)
against exp to 50 digits, and on the device bit for bit against the host."""
import ctypes
import math
import subprocess
from decimal import Decimal, getcontext
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
HARNESS = r"""
#include "yz_exp.h"
#include <cstdio>
#include <vector>
int main(int argc, char **argv)
{
	FILE *f = std::fopen(argv[1], "rb");
	std::vector<double> x;
	double v;
	while(std::fread(&v, sizeof v, 1, f) == 1) x.push_back(v);
	std::fclose(f);
	FILE *g = std::fopen(argv[2], "wb");
	for(double a : x) { const double y = yz::crexp::Exp(a); std::fwrite(&y, sizeof y, 1, g); }
	std::fclose(g);
	return 0;
}
"""


def arguments():
    rng = np.random.default_rng(7)
    special = [0.0, -0.0, 1.0, -1.0, 0.5 * math.log(2), -0.5 * math.log(2), 709.7, -707.9, 1e-300, -1e-300,
               2.0 ** -60, 10.0 * (0.3 - 0.5), -7.0 * (0.7 - 0.5)]
    return np.concatenate([np.array(special), rng.uniform(-12, 12, 12000), rng.uniform(-700, 700, 3000),
                           rng.uniform(-1e-3, 1e-3, 2000)])


def host_exp(tmp_path, x):
    src = tmp_path / "h.cpp"
    src.write_text(HARNESS)
    exe = tmp_path / "h"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(REPO / "yuzen_b200" / "csrc"),
                    str(src), "-o", str(exe)], check=True)
    x.astype("<f8").tofile(tmp_path / "x.bin")
    subprocess.run([str(exe), str(tmp_path / "x.bin"), str(tmp_path / "y.bin")], check=True)
    return np.fromfile(tmp_path / "y.bin", "<f8")


def test_correctly_rounded_on_the_host(tmp_path):
    getcontext().prec = 50
    x = arguments()
    y = host_exp(tmp_path, x)
    for a, b in zip(x, y):
        t = Decimal(float(a)).exp()
        b = float(b)
        for v in (math.nextafter(b, math.inf), math.nextafter(b, -math.inf)):
            assert abs(Decimal(b) - t) <= abs(Decimal(v) - t), (a, b)


@pytest.mark.gpu
def test_device_equals_host(tmp_path):
    import yuzen_b200 as yz
    x = arguments()
    yh = host_exp(tmp_path, x)
    L = yz.lib()
    L.yz_exp_cr.argtypes = [ctypes.c_longlong, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    yd = np.zeros_like(x)
    assert L.yz_exp_cr(len(x), x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                       yd.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    assert np.array_equal(yd.view(np.int64), yh.view(np.int64))
