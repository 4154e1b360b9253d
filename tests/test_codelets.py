"""The in-register DFT codelets (wavesim_b200/csrc/ws_codelets.cuh), on the
host: the committed header is what gen_codelets.py writes, and every
Dft<R, INV> agrees with numpy's FFT (sign -1 forward, +1 unnormalised
inverse: MATLAB's fft / ifft * R, which the reference's fftn/ifftn calls in
WaveSimBase.m:118-124 rest on)."""
import os
import shutil
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "wavesim_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"


def _radices():
    sys.path.insert(0, CSRC)
    try:
        import gen_codelets
        return list(gen_codelets.RADICES)
    finally:
        sys.path.pop(0)


def test_header_is_generated():
    out = subprocess.run([sys.executable, os.path.join(CSRC, "gen_codelets.py")], capture_output=True, text=True,
                         check=True).stdout
    with open(os.path.join(CSRC, "ws_codelets.cuh")) as f:
        assert f.read() == out


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.isdir(CUDA_INC), reason="needs g++ and CUDA headers")
def test_codelets_match_numpy(tmp_path):
    radices = _radices()
    calls = "\n".join(
        f"  if (R == {r}) {{ float2 v[{r}]; for (int i = 0; i < {r}; ++i) v[i] = make_float2(x[2*i], x[2*i+1]);"
        f" if (inv) ws::Dft<{r}, true>::run(v); else ws::Dft<{r}, false>::run(v);"
        f" for (int i = 0; i < {r}; ++i) std::printf(\"%.9g %.9g\\n\", v[i].x, v[i].y); }}" for r in radices)
    src = tmp_path / "cod.cpp"
    src.write_text(f"""#include <math.h>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#include "ws_codelets.cuh"
int main(int argc, char** argv) {{
  const int R = std::atoi(argv[1]), inv = std::atoi(argv[2]);
  float x[64];
  for (int i = 0; i < 2 * R; ++i) x[i] = (float)std::atof(argv[3 + i]);
{calls}
  return 0;
}}
""")
    exe = tmp_path / "cod"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", CSRC, "-I", CUDA_INC, str(src), "-o", str(exe)], check=True)
    rng = np.random.default_rng(14)
    for r in radices:
        for inv in (0, 1):
            x = (rng.standard_normal(r) + 1j * rng.standard_normal(r)).astype(np.complex64)
            args = [str(exe), str(r), str(inv)] + [f"{v:.9g}" for c in x for v in (c.real, c.imag)]
            out = subprocess.run(args, capture_output=True, text=True, check=True).stdout.split()
            got = np.array(out, dtype=np.float64).reshape(r, 2) @ np.array([1, 1j])
            want = np.fft.ifft(x.astype(np.complex128)) * r if inv else np.fft.fft(x.astype(np.complex128))
            assert np.max(np.abs(got - want)) < 2e-6 * np.sqrt(r) * np.max(np.abs(want)), (r, inv)
