"""The C ABI from a C host (no GPU needed): include/ffroom.h compiles as C11
and a C program linked against libffroom_cuda.so builds a room, sizes it,
submits it to the server and gets its outcome back (on a box without a GPU
the outcome carries the handle's CUDA error; with one, the finished run)."""
import os
import subprocess

import pytest

from conftest import ROOT

PKG = os.path.join(ROOT, "ff-room_b200")

SRC = r"""
#include <stdio.h>
#include <stdlib.h>
#include "ffroom.h"

int main(void)
{
    enum { NX = 12, NY = 10, NZ = 8 };
    static double dx[NX], dy[NY], dz[NZ];
    static uint8_t ct[NX * NY * NZ];
    for (int i = 0; i < NX; i++) dx[i] = 0.25;
    for (int j = 0; j < NY; j++) dy[j] = 0.25;
    for (int k = 0; k < NZ; k++) dz[k] = 0.25;
    /* a fan cell on the west wall, an outflow plane on the east wall */
    ffr_fan fan = {1, 1, 4, 5, 3, 4, {1.0, 0.0, 0.0}};
    for (int j = 4; j <= 5; j++)
        for (int k = 3; k <= 4; k++) ct[(1 * NY + j) * NZ + k] = FFR_INFLOW;
    for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++) ct[((NX - 1) * NY + j) * NZ + k] = FFR_OUTFLOW;
    ffr_patch out = {0, 1, 0, NY - 1, 0, NZ - 1, 0, 0.0};
    ffr_room_desc room = {NX, NY, NZ, 3.0, 2.5, 2.0, dx, dy, dz, ct, 1, &fan, 1, &out, 0, NULL};
    ffr_fluid_params p = {1.2, 1.5e-5, 0.01, 4, 1e-4, 200, 1e-6, FFR_UPWIND1, 0, 0, 20.0, 1e30, 0,
                          9.81, 1.0 / 293.15, 0.026, 1005.0, FFR_PREC_MIXED, FFR_POISSON_MGPCG};
    size_t bytes = 0;
    if (ffr_fluid_estimate_bytes(&room, &p, &bytes) != FFR_OK || bytes == 0) return 2;
    ffr_server *srv = NULL;
    if (ffr_server_create(64 * bytes, 4, 2, &srv) != FFR_OK) return 3;
    if (ffr_server_submit(srv, 42, &room, &p, 4) != FFR_OK) return 4;
    ffr_outcome o[4];
    int n = 0;
    if (ffr_server_drain(srv, o, 4, &n) != FFR_OK || n != 1) return 5;
    printf("%lld %lld %d %d %zu %s\n", o[0].id, o[0].cells, o[0].status, o[0].steps, bytes,
           ffr_status_string(o[0].status));
    ffr_server_destroy(srv);
    return 0;
}
"""


def test_c_program_drives_the_server(tmp_path):
    lib = os.path.join(PKG, "libffroom_cuda.so")
    if not os.path.exists(lib):
        pytest.skip("libffroom_cuda.so is not built")
    src = tmp_path / "host.c"
    src.write_text(SRC)
    exe = tmp_path / "host"
    subprocess.check_call(["gcc", "-std=c11", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                           "-L", PKG, "-lffroom_cuda", f"-Wl,-rpath,{PKG}", "-o", str(exe)])
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    rid, cells, status, steps, nbytes = r.stdout.split()[:5]
    assert (int(rid), int(cells)) == (42, 12 * 10 * 8) and int(nbytes) > 0
    assert (int(status) == 0 and int(steps) == 4) or (int(status) != 0 and int(steps) == 0)
