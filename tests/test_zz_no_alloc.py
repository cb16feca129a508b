"""sw_compute_block_static: the block handler for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc (a host whose GPU memory all belongs to its own pool
allocator, a plug-in whose process has a fixed device-memory budget).
The static entry point runs the same plain block kernel as sw_compute_block_device with its
scratch in the library's own device array.  It must give the same Int16 distances as the
allocating entry point (exact equality), on two calls in a row (the second reuses the array
the first left behind), and the second call must not change the device's free memory (the first
may: loading the library's device image on first use places the array).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cfg(lib, matrix, o, e):
    cfg = lib.sw_config()
    cfg.mode, cfg.alignment_type, cfg.distance_fn = lib.SW_MODE_SWG_MPI, lib.SW_NUCLEIC, 0
    cfg.gap_open, cfg.gap_extension = float(o), float(e)
    C.memmove(cfg.scores, matrix.Scores.ctypes.data, 128 * 128 * 2)
    cfg.device, cfg.lanes = 0, 0
    return cfg


def test_static_block_handler_matches_allocating_one_twice():
    import torch
    import csharp_b200 as cs
    from csharp_b200 import build, lib, synth
    build.build()
    rng = np.random.default_rng(31)
    lens = np.concatenate([rng.integers(1, 400, 70), [0, 1, 900]])
    seqs = [s.tobytes() for s in synth.dna_family(len(lens), 5, lens, seed=41)]
    N = len(seqs)
    matrix = cs.ScoringMatrix.Load("EDNAFULL")
    eng = cs.Engine(matrix, 16, 4).upload(seqs)  # the allocating entry point, for the expected values
    concat, off = cs.pack_sequences(seqs)
    d_seq = torch.from_numpy(concat).cuda()
    d_off = torch.from_numpy(off).cuda()
    cfg = _cfg(lib, matrix, 16, 4)
    blocks = [(0, N - 1, 0, N - 1, 1), (40, 72, 3, 30, 0)]
    L = lib.load()
    for call, (rs, re_, cs_, ce, diag) in enumerate(blocks):
        R, Cc = re_ - rs + 1, ce - cs_ + 1
        want = torch.zeros((R, Cc), dtype=torch.int16, device="cuda")
        eng.compute_block_device(rs, re_, cs_, ce, diag, want.data_ptr(), Cc)
        eng.synchronize()
        got = torch.zeros((R, Cc), dtype=torch.int16, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        n = C.c_int64()
        rc = L.sw_compute_block_static(C.byref(cfg), C.c_void_p(d_seq.data_ptr()), C.c_void_p(d_off.data_ptr()), N,
                                       rs, re_, cs_, ce, diag, C.c_void_p(got.data_ptr()), Cc, C.byref(n), None)
        assert rc == lib.SW_OK
        torch.cuda.synchronize()
        expected_pairs = R * (R - 1) // 2 if diag else R * Cc
        assert n.value == expected_pairs
        np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy())
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before


def test_static_block_handler_rejects_out_of_table_residues():
    import torch
    import csharp_b200 as cs
    from csharp_b200 import lib
    concat, off = cs.pack_sequences([b"ACGT", bytes([65, 200, 67])])
    d_seq = torch.from_numpy(concat).cuda()
    d_off = torch.from_numpy(off).cuda()
    out = torch.zeros((2, 2), dtype=torch.int16, device="cuda")
    cfg = _cfg(lib, cs.ScoringMatrix.Load("EDNAFULL"), 16, 4)
    n = C.c_int64()
    rc = lib.load().sw_compute_block_static(C.byref(cfg), C.c_void_p(d_seq.data_ptr()), C.c_void_p(d_off.data_ptr()), 2,
                                            0, 1, 0, 1, 1, C.c_void_p(out.data_ptr()), 2, C.byref(n), None)
    assert rc == lib.SW_E_ARG
