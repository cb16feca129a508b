"""sw_compute_block_static: the block handler for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc (a host whose GPU memory all belongs to its own pool
allocator, a plug-in whose process has a fixed device-memory budget).
The static entry point runs the same plain block kernel as sw_compute_block_device with its
scratch in the library's own device array.  It must give the same Int16 distances as the
allocating entry point (exact equality) in every mode and alphabet, on two calls in a row (the
second reuses the array the first left behind), on the legacy stream and on a caller's stream,
and the second call must not change the device's free memory (the first may: loading the
library's device image on first use places the array).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = {"mpi": 0, "ms": 1, "nw": 2}


def _cfg(lib, matrix, o, e, mode=0, protein=False, dist=0, device=0):
    cfg = lib.sw_config()
    cfg.mode, cfg.alignment_type, cfg.distance_fn = mode, lib.SW_PROTEIN if protein else lib.SW_NUCLEIC, dist
    cfg.gap_open, cfg.gap_extension = float(o), float(e)
    C.memmove(cfg.scores, matrix.Scores.ctypes.data, 128 * 128 * 2)
    cfg.device, cfg.lanes = device, 0
    return cfg


def _seqs(protein, n_extra):
    from csharp_b200 import synth
    import csharp_b200 as cs
    rng = np.random.default_rng(31 + n_extra)
    lens = np.concatenate([rng.integers(1, 400, 70), [0, 1, 900]])
    if protein:
        bl = cs.ScoringMatrix.Load("BLOSUM62").Scores
        return [s.tobytes() for s in synth.protein_family(len(lens), 5, np.maximum(lens, 1), 41, bl)] + [b""]
    return [s.tobytes() for s in synth.dna_family(len(lens), 5, lens, seed=41)]


def _static(L, cfg, d_seq, d_off, N, blk, out, stream=None):
    rs, re_, cs_, ce, diag = blk
    n = C.c_int64()
    rc = L.sw_compute_block_static(C.byref(cfg), C.c_void_p(d_seq.data_ptr()), C.c_void_p(d_off.data_ptr()), N,
                                   rs, re_, cs_, ce, diag, C.c_void_p(out.data_ptr()), out.shape[1], C.byref(n),
                                   C.c_void_p(stream) if stream else None)
    return rc, n.value


@pytest.mark.parametrize("mode,matrix", [("mpi", "EDNAFULL"), ("ms", "EDNAFULL"), ("nw", "EDNAFULL"),
                                         ("mpi", "BLOSUM62"), ("ms", "BLOSUM62"), ("nw", "BLOSUM62")])
def test_static_block_handler_matches_allocating_one_twice(mode, matrix):
    import torch
    import csharp_b200 as cs
    from csharp_b200 import build, lib
    build.build()
    protein = matrix == "BLOSUM62"
    seqs = _seqs(protein, len(mode))
    N = len(seqs)
    m = cs.ScoringMatrix.Load(matrix)
    o, e = (10, 1) if protein else (16, 4)
    eng = cs.Engine(m, o, e, mode=MODES[mode], alignment_type=cs.PROTEIN if protein else cs.NUCLEIC).upload(seqs)
    concat, off = cs.pack_sequences(seqs)
    d_seq = torch.from_numpy(concat).cuda()
    d_off = torch.from_numpy(off).cuda()
    cfg = _cfg(lib, m, o, e, MODES[mode], protein)
    blocks = [(0, N - 1, 0, N - 1, 1), (40, N - 1, 3, 30, 0)]
    L = lib.load()
    side = torch.cuda.Stream()
    for call, blk in enumerate(blocks):
        rs, re_, cs_, ce, diag = blk
        R, Cc = re_ - rs + 1, ce - cs_ + 1
        want = torch.zeros((R, Cc), dtype=torch.int16, device="cuda")
        eng.compute_block_device(rs, re_, cs_, ce, diag, want.data_ptr(), Cc)
        eng.synchronize()
        got = torch.zeros((R, Cc), dtype=torch.int16, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc, n = _static(L, cfg, d_seq, d_off, N, blk, got, stream=side.cuda_stream if call else None)
        assert rc == lib.SW_OK
        torch.cuda.synchronize()
        tri = diag and mode != "ms"
        assert n == (R * (R - 1) // 2 if tri else R * Cc)
        np.testing.assert_array_equal(got.cpu().numpy(), want.cpu().numpy())
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before
    eng.close()


def test_static_block_handler_rejects_bad_inputs():
    import torch
    import csharp_b200 as cs
    from csharp_b200 import lib
    L = lib.load()
    m = cs.ScoringMatrix.Load("EDNAFULL")
    concat, off = cs.pack_sequences([b"ACGT", bytes([65, 200, 67])])
    d_seq = torch.from_numpy(concat).cuda()
    d_off = torch.from_numpy(off).cuda()
    out = torch.zeros((2, 2), dtype=torch.int16, device="cuda")
    blk = (0, 1, 0, 1, 1)
    assert _static(L, _cfg(lib, m, 16, 4), d_seq, d_off, 2, blk, out)[0] == lib.SW_E_ARG  # residue 200
    # a sequence beyond the array's 16,383-residue limit is refused before any alignment
    long_c, long_o = cs.pack_sequences([b"ACGT", b"A" * 16384])
    d_long, d_loff = torch.from_numpy(long_c).cuda(), torch.from_numpy(long_o).cuda()
    assert _static(L, _cfg(lib, m, 16, 4), d_long, d_loff, 2, blk, out)[0] == lib.SW_E_UNSUPPORTED
    ok_c, ok_o = cs.pack_sequences([b"ACGT", b"ACGA"])
    d_ok, d_okoff = torch.from_numpy(ok_c).cuda(), torch.from_numpy(ok_o).cuda()
    assert _static(L, _cfg(lib, m, 16, 4, dist=7), d_ok, d_okoff, 2, blk, out)[0] == lib.SW_E_ARG
    assert _static(L, _cfg(lib, m, 16, 4, dist=1), d_ok, d_okoff, 2, blk, out)[0] == lib.SW_E_UNSUPPORTED
    # buffers that are not the configured device's memory, or a device that does not exist
    host_out = torch.zeros((2, 2), dtype=torch.int16)
    assert _static(L, _cfg(lib, m, 16, 4), d_ok, d_okoff, 2, blk, host_out)[0] == lib.SW_E_ARG
    before = torch.cuda.current_device()
    bad_dev = torch.cuda.device_count()
    assert _static(L, _cfg(lib, m, 16, 4, device=bad_dev), d_ok, d_okoff, 2, blk, out)[0] == lib.SW_E_ARG
    assert torch.cuda.current_device() == before
    assert _static(L, _cfg(lib, m, 16, 4), d_ok, d_okoff, 2, blk, out)[0] == lib.SW_OK
    torch.cuda.synchronize()
