"""Autotuner of launch shapes: the cache table, its JSON file and the mode, through
the C ABI (no GPU needed: these calls touch no device).

The GPU side (every candidate a key may pick passing the same oracle checks, and a
measurement in MEASURE mode) is in test_autotune_gpu.py."""
import ctypes
import json
import os
import subprocess
import sys

import pytest

import c7x_dsplib_b200 as D

OFF, CACHED, MEASURE = 0, 1, 2
INVALID_VALUE = 2


@pytest.fixture
def table():
    """The process-wide table, emptied and back in CACHED mode with no file afterwards."""
    L = D.lib()
    L.DSPLIB_gpu_autotuneSetCachePath(None)
    L.DSPLIB_gpu_autotuneClear()
    yield L
    L.DSPLIB_gpu_autotuneSetCachePath(None)
    L.DSPLIB_gpu_autotuneClear()
    L.DSPLIB_gpu_autotuneSetMode(CACHED)


def test_store_lookup_clear(table):
    L = table
    assert L.DSPLIB_gpu_autotuneLookup(b"fir_bf16x3|T=256|tiles=2^3|batch=2^10|nch=1|sms=148") == -1
    assert L.DSPLIB_gpu_autotuneStore(b"fir_bf16x3|T=256|tiles=2^3|batch=2^10|nch=1|sms=148", 4) == 0
    assert L.DSPLIB_gpu_autotuneStore(b"bq_scan|form=1|S=4|nch=0|ch=2^5|N=2^13|sms=148", 1604) == 0
    assert L.DSPLIB_gpu_autotuneLookup(b"fir_bf16x3|T=256|tiles=2^3|batch=2^10|nch=1|sms=148") == 4
    assert L.DSPLIB_gpu_autotuneCount() == 2
    # overwrite, invalid entries refused
    assert L.DSPLIB_gpu_autotuneStore(b"bq_scan|form=1|S=4|nch=0|ch=2^5|N=2^13|sms=148", 808) == 0
    assert L.DSPLIB_gpu_autotuneLookup(b"bq_scan|form=1|S=4|nch=0|ch=2^5|N=2^13|sms=148") == 808
    assert L.DSPLIB_gpu_autotuneStore(b"k", -1) == INVALID_VALUE
    assert L.DSPLIB_gpu_autotuneStore(b"", 3) == INVALID_VALUE
    assert L.DSPLIB_gpu_autotuneStore(None, 3) == INVALID_VALUE
    assert L.DSPLIB_gpu_autotuneLookup(None) == -1
    assert L.DSPLIB_gpu_autotuneClear() == 0
    assert L.DSPLIB_gpu_autotuneCount() == 0


def test_cache_file_roundtrip(table, tmp_path):
    L = table
    path = tmp_path / "tune.json"
    assert L.DSPLIB_gpu_autotuneSave() == INVALID_VALUE  # no file set
    assert L.DSPLIB_gpu_autotuneSetCachePath(str(path).encode()) == 0  # absent file: nothing loaded
    assert L.DSPLIB_gpu_autotuneCount() == 0
    entries = {"fir_int|dtype=0|q=1|T=128|tiles=2^3|batch=2^12|sms=148": 66,
               "bank_runs|ch=2^11|samples=2^27|Tmax=512|sms=148": 8,
               "bq_scan|form=3|S=4|nch=1|ch=2^12|N=2^13|sms=148": 1602}
    for k, v in entries.items():
        assert L.DSPLIB_gpu_autotuneStore(k.encode(), v) == 0
    assert L.DSPLIB_gpu_autotuneSave() == 0
    doc = json.loads(path.read_text())
    assert doc["format"] == "dsplib_b200 autotune 1"
    assert doc["entries"] == entries
    # a fresh table reads them back
    L.DSPLIB_gpu_autotuneSetCachePath(None)
    L.DSPLIB_gpu_autotuneClear()
    assert L.DSPLIB_gpu_autotuneSetCachePath(str(path).encode()) == 0
    assert L.DSPLIB_gpu_autotuneCount() == 3
    for k, v in entries.items():
        assert L.DSPLIB_gpu_autotuneLookup(k.encode()) == v
    # merged with entries already in the table; the table's own win on a clash
    L.DSPLIB_gpu_autotuneSetCachePath(None)
    L.DSPLIB_gpu_autotuneClear()
    L.DSPLIB_gpu_autotuneStore(b"other|x=1|sms=148", 2)
    L.DSPLIB_gpu_autotuneSetCachePath(str(path).encode())
    assert L.DSPLIB_gpu_autotuneCount() == 4


@pytest.mark.parametrize("text", ["", "not json", '{"format": "something else", "entries": {"a": 1}}',
                                  '{"format": "dsplib_b200 autotune 1", "entries": {"a": }}',
                                  '{"format": "dsplib_b200 autotune 1", "entries": {"a": 1'])
def test_malformed_cache_file_ignored(table, tmp_path, text):
    L = table
    path = tmp_path / "bad.json"
    path.write_text(text)
    assert L.DSPLIB_gpu_autotuneSetCachePath(str(path).encode()) == 0
    assert L.DSPLIB_gpu_autotuneCount() == 0
    # saving replaces it with a well-formed file
    L.DSPLIB_gpu_autotuneStore(b"k|sms=1", 5)
    assert L.DSPLIB_gpu_autotuneSave() == 0
    assert json.loads(path.read_text())["entries"] == {"k|sms=1": 5}


def test_mode(table):
    L = table
    for m in (OFF, MEASURE, CACHED):
        assert L.DSPLIB_gpu_autotuneSetMode(m) == 0
        assert L.DSPLIB_gpu_autotuneGetMode() == m
    assert L.DSPLIB_gpu_autotuneSetMode(3) == INVALID_VALUE
    assert L.DSPLIB_gpu_autotuneSetMode(-1) == INVALID_VALUE
    assert L.DSPLIB_gpu_autotuneGetMode() == CACHED


def test_handle_queries_need_an_initialised_handle(table):
    L = table
    buf = ctypes.create_string_buffer(64)
    assert L.DSPLIB_gpu_autotuneHandleKey(None, buf, 64) == 0
    assert buf.value == b""
    assert L.DSPLIB_gpu_autotuneHandleCandidate(None, 0) == -1
    assert L.DSPLIB_gpu_autotune(None) == 5  # DSPLIB_ERR_NULL_POINTER
    h = D.FirHandle()  # never initialised
    assert L.DSPLIB_gpu_autotuneHandleKey(h.h, buf, 64) == 0


def test_environment_sets_file_and_mode(tmp_path):
    """DSPLIB_GPU_TUNE_CACHE and DSPLIB_GPU_AUTOTUNE give a new process its settings."""
    path = tmp_path / "env.json"
    path.write_text(json.dumps({"format": "dsplib_b200 autotune 1", "entries": {"fir_bf16x3|T=64|sms=148": 2}}))
    code = ("import c7x_dsplib_b200 as D; L = D.lib(); "
            "print(L.DSPLIB_gpu_autotuneGetMode(), L.DSPLIB_gpu_autotuneLookup(b'fir_bf16x3|T=64|sms=148'))")
    env = dict(os.environ, DSPLIB_GPU_TUNE_CACHE=str(path), DSPLIB_GPU_AUTOTUNE="0")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert out.stdout.split() == ["0", "2"]
