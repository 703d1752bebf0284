"""Python mirror of IndexinGPU's gpu_masstree host API over libmt_b200.so.

Method names, argument order and meaning follow the reference's
GpuMasstree::gpu_masstree (include/gpu_masstree.hpp:84-191):

    find(keys, max_key_length, key_lengths, values, max_value_length,
         value_lengths, num_keys, stream=0)
    insert / update(keys, max_key_length, key_lengths, values,
         max_value_length, value_lengths, num_keys, stream=0)
    erase(keys, max_key_length, key_lengths, num_keys, stream=0)
    scan(lower_keys, lower_key_lengths, max_key_length, max_count_per_query,
         num_queries, upper_keys=None, upper_key_lengths=None, counts=None,
         values=None, max_value_length=1, value_lengths=None, out_keys=None,
         out_key_lengths=None, stream=0)
    mixed_batch(request_types, keys, max_key_length, key_lengths, values,
         max_value_length, value_lengths, results, num_requests, stream=0)

The reference's compile-time switches become keyword arguments
(concurrent=, update_if_exists=, use_upper_key=).  Buffers are torch tensors in
device memory or pinned host memory (or raw integer addresses); None means the
reference's nullptr.  Calls are asynchronous; sync() waits and raises on a
device-side error.
"""
import ctypes

from . import _lib

REQ_INSERT, REQ_ERASE, REQ_FIND, REQ_UPDATE = 0, 1, 2, 3
FLAG_CONCURRENT, FLAG_UPDATE_IF_EXISTS, FLAG_USE_UPPER_KEY, FLAG_SINGLE_PASS, FLAG_BUCKET_KEYS = 1, 2, 4, 8, 16
FLAG_PERSISTENT = 32
FLAG_MERGE = 64
FLAG_REMOVE_EMPTY_LAYERS = 128
FLAG_INPUTS_ON_STREAM = 256
FLAG_GROUP_BY_KEY = 512
STATUS = {0: "MT_OK", 1: "MT_ERR_OOM", 2: "MT_ERR_LOCK_TIMEOUT", 3: "MT_ERR_CORRUPT", 4: "MT_ERR_INVALID_ARG",
          5: "MT_ERR_CUDA", 6: "MT_ERR_RETRY_LIMIT", 7: "MT_ERR_KEY_TOO_LONG", 8: "MT_ERR_BATCH_TOO_LARGE"}


class MasstreeError(RuntimeError):
    def __init__(self, code, what, site=0):
        self.code = code
        self.site = site
        where = f" (detected at source file {site >> 16}, line {site & 0xFFFF})" if site else ""
        super().__init__(f"{what}: {STATUS.get(code, code)}{where}")


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x or None
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return x.ctypes.data  # numpy


def _stream(s):
    if s is None or s == 0:
        return None
    if isinstance(s, int):
        return s
    return s.cuda_stream  # torch.cuda.Stream


class GpuMasstree:
    """Ordered GPU index over variable-length u32-slice keys and values."""

    def __init__(self, pool_ratio=0.9, tile_size=8, pool_bytes=None):
        self._lib = _lib.load()
        h = ctypes.c_void_p()
        if pool_bytes is not None:
            rc = self._lib.mt_create_bytes(ctypes.byref(h), int(pool_bytes), tile_size)
        else:
            rc = self._lib.mt_create(ctypes.byref(h), float(pool_ratio), tile_size)
        self._check(rc, "mt_create")
        self._h = h

    # -- lifetime ---------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.mt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _check(rc, what):
        if rc != 0:
            raise MasstreeError(rc, what)

    # -- configuration ------------------------------------------------------------
    def set_tile_size(self, tile_size):
        self._check(self._lib.mt_set_tile_size(self._h, tile_size), "mt_set_tile_size")

    def set_write_tile_size(self, tile_size):
        self._check(self._lib.mt_set_write_tile_size(self._h, tile_size), "mt_set_write_tile_size")

    def set_scan_tile_size(self, tile_size):
        """Lanes per scan query (0: the find width)."""
        self._check(self._lib.mt_set_scan_tile_size(self._h, tile_size), "mt_set_scan_tile_size")

    def set_blocks_per_sm(self, blocks_per_sm):
        self._check(self._lib.mt_set_blocks_per_sm(self._h, blocks_per_sm), "mt_set_blocks_per_sm")

    def set_group_hash_bits(self, bits):
        """Bits of the key hash the grouped form of mixed_batches sorts by
        (default 64; fewer make different keys share a hash: for tests)."""
        self._check(self._lib.mt_set_group_hash_bits(self._h, bits), "mt_set_group_hash_bits")

    def set_upderase_tile_size(self, tile_size):
        """Lanes per update/erase of mixed batches (0: the write width)."""
        self._check(self._lib.mt_set_upderase_tile_size(self._h, tile_size), "mt_set_upderase_tile_size")

    def set_lock_wait(self, attempts):
        """Lock attempts before a waiting request reports MT_ERR_LOCK_TIMEOUT."""
        self._check(self._lib.mt_set_lock_wait(self._h, attempts), "mt_set_lock_wait")

    def inject_node_lock(self, slab, locked=True):
        """Test hook: set or clear the LOCK bit of node `slab` from the host."""
        self._check(self._lib.mt_inject_node_lock(self._h, slab, 1 if locked else 0), "mt_inject_node_lock")

    # -- host API (reference gpu_masstree.hpp:86-191) ----------------------------
    def find(self, keys, max_key_length, key_lengths, values, max_value_length, value_lengths, num_keys,
             stream=0, concurrent=False):
        rc = self._lib.mt_find(self._h, _ptr(keys), max_key_length, _ptr(key_lengths), _ptr(values),
                               max_value_length, _ptr(value_lengths), num_keys,
                               FLAG_CONCURRENT if concurrent else 0, _stream(stream))
        self._check(rc, "mt_find")

    def insert(self, keys, max_key_length, key_lengths, values, max_value_length, value_lengths, num_keys,
               stream=0, update_if_exists=False, results=None):
        rc = self._lib.mt_insert(self._h, _ptr(keys), max_key_length, _ptr(key_lengths), _ptr(values),
                                 max_value_length, _ptr(value_lengths), num_keys, _ptr(results),
                                 FLAG_UPDATE_IF_EXISTS if update_if_exists else 0, _stream(stream))
        self._check(rc, "mt_insert")

    def update(self, keys, max_key_length, key_lengths, values, max_value_length, value_lengths, num_keys,
               stream=0, results=None):
        rc = self._lib.mt_update(self._h, _ptr(keys), max_key_length, _ptr(key_lengths), _ptr(values),
                                 max_value_length, _ptr(value_lengths), num_keys, _ptr(results), 0,
                                 _stream(stream))
        self._check(rc, "mt_update")

    def erase(self, keys, max_key_length, key_lengths, num_keys, stream=0, results=None, merge=False,
              remove_empty_layers=False):
        flags = (FLAG_MERGE if merge else 0) | (FLAG_REMOVE_EMPTY_LAYERS if remove_empty_layers else 0)
        rc = self._lib.mt_erase(self._h, _ptr(keys), max_key_length, _ptr(key_lengths), num_keys, _ptr(results),
                                flags, _stream(stream))
        self._check(rc, "mt_erase")

    def scan(self, lower_keys, lower_key_lengths, max_key_length, max_count_per_query, num_queries,
             upper_keys=None, upper_key_lengths=None, counts=None, values=None, max_value_length=1,
             value_lengths=None, out_keys=None, out_key_lengths=None, stream=0, use_upper_key=None,
             concurrent=False):
        if use_upper_key is None:
            use_upper_key = upper_keys is not None
        flags = (FLAG_USE_UPPER_KEY if use_upper_key else 0) | (FLAG_CONCURRENT if concurrent else 0)
        rc = self._lib.mt_scan(self._h, _ptr(lower_keys), _ptr(lower_key_lengths), max_key_length,
                               max_count_per_query, num_queries, _ptr(upper_keys), _ptr(upper_key_lengths),
                               _ptr(counts), _ptr(values), max_value_length, _ptr(value_lengths), _ptr(out_keys),
                               _ptr(out_key_lengths), flags, _stream(stream))
        self._check(rc, "mt_scan")

    def mixed_batch(self, request_types, keys, max_key_length, key_lengths, values, max_value_length,
                    value_lengths, results, num_requests, stream=0, single_pass=False, bucket_keys=False,
                    merge=False, remove_empty_layers=False):
        flags = ((FLAG_SINGLE_PASS if single_pass else 0) | (FLAG_BUCKET_KEYS if bucket_keys else 0) |
                 (FLAG_MERGE if merge else 0) | (FLAG_REMOVE_EMPTY_LAYERS if remove_empty_layers else 0))
        rc = self._lib.mt_mixed_batch(self._h, _ptr(request_types), _ptr(keys), max_key_length, _ptr(key_lengths),
                                      _ptr(values), max_value_length, _ptr(value_lengths), _ptr(results),
                                      num_requests, flags, _stream(stream))
        self._check(rc, "mt_mixed_batch")

    def mixed_batch_host(self, request_types, keys, max_key_length, key_lengths, values, max_value_length,
                         value_lengths, results, num_requests, stream=0, chunk=0, bucket_keys=False,
                         inputs_on_stream=False):
        """mixed_batch with every buffer in (pinned) host memory; uploads, work and
        downloads of consecutive chunks overlap.  Asynchronous: sync(stream)
        before reading the results or reusing the buffers.  inputs_on_stream:
        the uploads wait for work already queued on `stream` (inputs it writes)."""
        flags = (FLAG_BUCKET_KEYS if bucket_keys else 0) | (FLAG_INPUTS_ON_STREAM if inputs_on_stream else 0)
        rc = self._lib.mt_mixed_batch_host(self._h, _ptr(request_types), _ptr(keys), max_key_length,
                                           _ptr(key_lengths), _ptr(values), max_value_length, _ptr(value_lengths),
                                           _ptr(results), num_requests, chunk, flags, _stream(stream))
        self._check(rc, "mt_mixed_batch_host")

    # -- many sub-batches in one call ------------------------------------------------
    def reserve_batches(self, max_subbatches, max_total_requests):
        self._check(self._lib.mt_batches_reserve(self._h, max_subbatches, max_total_requests), "mt_batches_reserve")

    def mixed_batches(self, descriptors, num_subbatches, max_key_length, max_value_length, stream=0,
                      bucket_keys=False, persistent=False, group_by_key=False):
        """Serve num_subbatches mixed batches in order (three class kernels per
        sub-batch on forked streams, or one persistent launch for all with
        persistent=True, or all at once with the requests on each key resolved
        in sub-batch order with group_by_key=True).  `descriptors` is a device
        tensor holding mt_subbatch records (see pack_subbatches)."""
        flags = ((FLAG_BUCKET_KEYS if bucket_keys else 0) | (FLAG_PERSISTENT if persistent else 0) |
                 (FLAG_GROUP_BY_KEY if group_by_key else 0))
        rc = self._lib.mt_mixed_batches(self._h, _ptr(descriptors), num_subbatches, max_key_length,
                                        max_value_length, flags, _stream(stream))
        self._check(rc, "mt_mixed_batches")

    # -- serving ---------------------------------------------------------------------
    def serve(self, types, keys, max_key_length, key_lengths, values, max_value_length, value_lengths, results,
              request_first_op, request_num_ops, arrival_ns, plain=False, chunk_ops=0, epoch_us=0,
              memory_budget=0.0, online=False):
        """Serve an open-loop request stream (mt_serve).  Op buffers are device
        tensors holding every request's ops; request_first_op, request_num_ops
        and arrival_ns (nanoseconds after the start, non-decreasing) are host
        arrays, one entry per request.  Returns (latency_ns numpy array, stats
        dict).  plain=True serves one synchronous mixed_batch per request;
        online=True takes HOST (pinned) op buffers and submits each request
        through the online server API at its arrival time."""
        import numpy as np
        first = np.ascontiguousarray(request_first_op, dtype=np.uint32)
        nops = np.ascontiguousarray(request_num_ops, dtype=np.uint32)
        arr = np.ascontiguousarray(arrival_ns, dtype=np.uint64)
        n = len(first)
        if len(nops) != n or len(arr) != n:
            raise ValueError("request arrays differ in length")
        lat = np.zeros(n, dtype=np.uint64)
        plan = _lib.MtServePlan()
        plan.types, plan.keys, plan.key_lengths = _ptr(types), _ptr(keys), _ptr(key_lengths)
        plan.values, plan.value_lengths, plan.results = _ptr(values), _ptr(value_lengths), _ptr(results)
        plan.max_key_length, plan.max_value_length = max_key_length, max_value_length
        plan.request_first_op = first.ctypes.data
        plan.request_num_ops = nops.ctypes.data
        plan.arrival_ns = arr.ctypes.data
        plan.num_requests = n
        plan.mode = 1 if plain else (2 if online else 0)
        plan.chunk_ops, plan.epoch_us, plan.memory_budget = chunk_ops, epoch_us, memory_budget
        st = _lib.MtServeStats()
        rc = self._lib.mt_serve(self._h, ctypes.byref(plan), lat.ctypes.data, ctypes.byref(st))
        self._check(rc, "mt_serve")
        out = {f: getattr(st, f) for f, _ in _lib.MtServeStats._fields_ if f != "stage_ns"}
        out["stage_ns"] = dict(zip(("queued", "upload", "device", "deliver"), (int(x) for x in st.stage_ns)))
        return lat, out

    # -- status ---------------------------------------------------------------------
    def sync(self, stream=0):
        """Wait for the stream; raise MasstreeError if a device error was recorded."""
        rc = self._lib.mt_sync(self._h, _stream(stream))
        if rc != 0:
            site = self.stats()["device_error_site"] if rc != 5 else 0
            raise MasstreeError(rc, "device", site)

    def reclaim(self, stream=0):
        self._check(self._lib.mt_reclaim(self._h, _stream(stream)), "mt_reclaim")

    def validate(self):
        """Structural check of the whole index; returns (ok, num_keys, report)."""
        n = ctypes.c_uint64()
        buf = ctypes.create_string_buffer(512)
        rc = self._lib.mt_validate(self._h, ctypes.byref(n), buf, 512)
        if rc not in (0, 3):
            self._check(rc, "mt_validate")
        return rc == 0, int(n.value), buf.value.decode()

    def stats(self):
        s = _lib.MtStats()
        self._check(self._lib.mt_stats(self._h, ctypes.byref(s)), "mt_stats")
        return {f: getattr(s, f) for f, _ in _lib.MtStats._fields_}


class MasstreeServer:
    """Online serving of a tree (mt_server_*): submit requests from host
    buffers while the device loop runs, poll their tickets, stop."""

    def __init__(self, tree, max_key_length, max_value_length, max_ops_in_flight=0, max_requests_in_flight=0,
                 chunk_ops=0, epoch_us=0, memory_budget=0.0):
        self._lib = tree._lib
        cfg = _lib.MtServerConfig(max_key_length, max_value_length, max_ops_in_flight, max_requests_in_flight,
                                  chunk_ops, epoch_us, memory_budget, 0)
        h = ctypes.c_void_p()
        rc = self._lib.mt_server_start(tree._h, ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise MasstreeError(rc, "mt_server_start")
        self._h = h

    def submit(self, types, keys, key_lengths, values, value_lengths, results, num_ops):
        """Queue one request; buffers are host memory (pinned tensors or numpy
        arrays, or integer addresses) that must stay untouched until done."""
        t = ctypes.c_uint64()
        rc = self._lib.mt_server_submit(self._h, _ptr(types), _ptr(keys), _ptr(key_lengths), _ptr(values),
                                        _ptr(value_lengths), _ptr(results), num_ops, ctypes.byref(t))
        if rc != 0:
            raise MasstreeError(rc, "mt_server_submit")
        return t.value

    def poll(self, ticket):
        """(done, latency_ns) of a ticket."""
        d, lat = ctypes.c_int(), ctypes.c_uint64()
        rc = self._lib.mt_server_poll(self._h, ticket, ctypes.byref(d), ctypes.byref(lat))
        if rc != 0:
            raise MasstreeError(rc, "mt_server_poll")
        return bool(d.value), int(lat.value)

    def stats(self):
        """Stage sums of the requests completed so far (mt_server_stats_t)."""
        st = _lib.MtServerStats()
        rc = self._lib.mt_server_stats(self._h, ctypes.byref(st))
        if rc != 0:
            raise MasstreeError(rc, "mt_server_stats")
        return {f: int(getattr(st, f)) for f, _ in _lib.MtServerStats._fields_ if f != "reserved"}

    def stop(self):
        if self._h:
            h, self._h = self._h, None
            rc = self._lib.mt_server_stop(h)
            if rc != 0:
                raise MasstreeError(rc, "mt_server_stop")


def line_atomicity_selftest(tile_size, nlines=64, iters=20000):
    """(reads, torn reads) of the 128-byte line-atomicity self-test."""
    lib = _lib.load()
    r, t = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib.mt_selftest_line_atomicity(tile_size, nlines, iters, ctypes.byref(r), ctypes.byref(t))
    if rc != 0:
        raise MasstreeError(rc, "mt_selftest_line_atomicity")
    return int(r.value), int(t.value)


def pack_subbatches(subbatches):
    """Pack sub-batches (dicts of device tensors: types, keys, lens, vals, vlens,
    results; lens and results may be None) into the mt_subbatch layout; returns
    a uint8 numpy array of 56 bytes per sub-batch, to be copied to the device."""
    import numpy as np
    rec = np.dtype([("types", "<u8"), ("keys", "<u8"), ("lens", "<u8"), ("vals", "<u8"), ("vlens", "<u8"),
                    ("results", "<u8"), ("n", "<u4"), ("reserved", "<u4")])
    arr = np.zeros(len(subbatches), dtype=rec)
    for i, sb in enumerate(subbatches):
        for f in ("types", "keys", "lens", "vals", "vlens", "results"):
            arr[i][f] = _ptr(sb.get(f)) or 0
        arr[i]["n"] = int(sb["n"])
    return arr.view(np.uint8)
