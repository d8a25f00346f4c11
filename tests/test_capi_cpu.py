"""CPU checks of the C-ABI boundary: the library loads, exports every symbol
include/utlpfor.h declares, and its host-side header helpers (BlockLength,
Header, MaxBlockLength*) agree with the oracle on valid and corrupt input.
No GPU call is made here."""
import json
import os
import re

import numpy as np
import pytest

import oracle_ref as O
from gen import KINDS32, KINDS64, block_values, block_values64

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "golden.json")))


@pytest.fixture(scope="module")
def U():
    from utlpfor_b200.build import build
    build()
    import utlpfor_b200 as U
    return U


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "utlpfor.h")).read()
    return sorted(set(re.findall(r"^UTL_API [^(]*?\b(utl_\w+)\(", src, re.M)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 30
    for must in ("utl_pack_u32", "utl_unpack_u32", "utl_get_u32", "utl_block_length", "utl_header",
                 "utl_pack_u64", "utl_unpack_u64", "utl_get_u64", "utl_pack_batch_u32", "utl_unpack_batch_u32",
                 "utl_get_batch_u32", "utl_codec_new"):
        assert must in names


def test_library_exports_every_declared_symbol(U):
    import ctypes
    from utlpfor_b200._lib import LIB_PATH, SIGNATURES
    lib = ctypes.CDLL(LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name
    bound = {s[0] for s in SIGNATURES}
    assert set(declared_symbols()) == bound


def test_max_block_length(U):
    for f in range(64):
        assert U.MaxBlockLength32(f) == O.max_block_length32(f)
        assert U.MaxBlockLength64(f) == O.max_block_length64(f)


def corrupted(rng, b):
    out = [b[:i] for i in range(0, min(len(b), 12))]
    for _ in range(30):
        x = bytearray(b)
        for _ in range(2):
            x[int(rng.integers(0, min(len(x), 12)))] ^= int(rng.integers(1, 256))
        out.append(bytes(x))
    return out


def test_block_length_and_header_match_oracle(U):
    rng = np.random.default_rng(8)
    blocks = [bytes.fromhex(g["packed_hex"]) for g in GOLDEN["golden_blocks"]]
    for flag in (0, 1, 2, 4, 5, 8):
        for kind in KINDS32:
            blocks.append(O.pack_u32(flag, block_values(rng, int(rng.integers(1, 129)), kind))[0])
        for kind in KINDS64:
            blocks.append(O.pack_u64(flag, block_values64(rng, int(rng.integers(1, 129)), kind))[0])
    for case in GOLDEN["fuzz_corpus"]:
        blocks.append(bytes(case["args"][0]))
    for b in blocks:
        for data in [b] + corrupted(rng, b):
            bl, err = O.block_length(data)
            try:
                got, gerr = U.BlockLength(data), 0
            except U.UTLError as e:
                got, gerr = 0, e.code
            assert (got, gerr) == (bl, err)
            fields, err = O.header(data)
            try:
                h, herr = U.Header(data), 0
            except U.UTLError as e:
                h, herr = None, e.code
            assert herr == err
            if err == 0:
                assert [int(x) for x in h] == fields


def test_no_cpu_fallback_without_gpu(U):
    """On a machine without a usable GPU the compute entry points fail with
    UTL_ERR_CUDA instead of computing on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(U.UTLError) as ei:
        U.PackUint32(0, [1, 2, 3])
    assert ei.value.code == -1 or "CUDA" in str(ei.value)
