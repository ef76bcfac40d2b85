"""The face-tile geometry of the TMA-staged momentum solve, checked on the CPU.

roundabout_b200/csrc/vphys_tiles.cuh is compiled here as plain C++ and, for
every tile of both face families on a range of grid shapes (odd and even nx,
ny, single rows and columns), every face's two cells are checked: they are
the cells the reference's clamping names (rdb_ocean_vdiff.F90:1665-1679),
and their offsets inside the staged blocks lie in [0, MT_BW) -- the blocks'
first elements are even, as a tiled TMA copy of doubles requires.  So the
kernel never reads a shared-memory element outside the block it staged.
"""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "roundabout_b200" / "csrc"

PROGRAM = r'''
#include <cstdio>
#include "vphys_tiles.cuh"
using namespace vphys;
int main() {
    const int shapes[][2] = {{1440, 1080}, {1, 1}, {2, 3}, {3, 2}, {127, 5}, {128, 4}, {129, 7}, {300, 1},
                             {1, 300}, {255, 9}, {256, 2}, {1441, 3}, {64, 64}, {33, 17}};
    long long checked = 0;
    for (auto &sh : shapes) {
        const int nx = sh[0], ny = sh[1];
        for (int fam = 0; fam < 2; ++fam) {
            const bool xf = fam == 0;
            const long long nf = xf ? (long long)(nx + 1) * ny : (long long)nx * (ny + 1);
            for (long long f0 = 0; f0 < nf; f0 += MT_TW) {
                const FaceTile t = face_tile(xf, f0, nx);
                if ((t.xa & 1) || (t.xb & 1) || (t.xw & 1)) { printf("odd start nx=%d ny=%d f0=%lld\n", nx, ny, f0); return 1; }
                for (long long f = f0; f < f0 + MT_TW && f < nf; ++f) {
                    const FaceCells c = face_cells(xf, f, nx, ny, t);
                    long long i, j, cl, cr;
                    if (xf) { j = f / (nx + 1); i = f - j * (nx + 1);
                        cl = (i - 1 > 0 ? i - 1 : 0) + (long long)nx * j; cr = (i < nx - 1 ? i : nx - 1) + (long long)nx * j; }
                    else { j = f / nx; i = f - j * nx;
                        cl = i + (long long)nx * (j - 1 > 0 ? j - 1 : 0); cr = i + (long long)nx * (j < ny - 1 ? j : ny - 1); }
                    const long long bl = c.bl ? t.xb : t.xa, br = c.br ? t.xb : t.xa;
                    if (c.cl != cl || c.cr != cr || bl + c.ol != cl || br + c.orr != cr || c.ol < 0 || c.ol >= MT_BW ||
                        c.orr < 0 || c.orr >= MT_BW || (xf && (c.bl || c.br))) {
                        printf("bad nx=%d ny=%d fam=%d f=%lld: ol=%d or=%d bl=%d br=%d\n", nx, ny, fam, f, c.ol, c.orr, c.bl, c.br);
                        return 1;
                    }
                    ++checked;
                }
            }
        }
    }
    printf("checked %lld faces\n", checked);
    return 0;
}
'''


def test_face_tile_offsets_in_bounds(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    src = tmp_path / "tiles.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "tiles"
    r = subprocess.run(["g++", "-O2", "-std=c++17", f"-I{CSRC}", "-o", str(exe), str(src)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "checked" in r.stdout
