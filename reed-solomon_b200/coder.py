"""Python mirror of the tape-reed-solomon coder API over the rs_b200 C ABI.

Class and method names, argument meaning and error behaviour follow the reference
crate (src/reedsolomon.rs, src/reedsolomon16.rs, src/errors.rs): `ReedSolomon(k, m)`
raises `RsError` carrying the same variant names the Rust `Error` enum uses. Shards
are any writable buffers (numpy uint8 arrays, bytearrays); reconstruct takes the
reference's two shard forms: `(buffer, present)` pairs, or `None` for an absent shard
that the call allocates (`Option<T>`, src/reedsolomon.rs:88-101).

Device-resident variants (`*_dev`) take CUDA tensors (anything with `data_ptr()`) or
integer device pointers, and a CUDA stream handle (an int; 0 = legacy default).
"""
import ctypes

import numpy as np

from . import _lib

ERROR_NAMES = {
    1: "TooFewShards",
    2: "TooManyShards",
    3: "TooFewDataShards",
    4: "TooManyDataShards",
    5: "TooFewParityShards",
    6: "TooManyParityShards",
    7: "TooFewBufferShards",
    8: "TooManyBufferShards",
    9: "IncorrectShardSize",
    10: "TooFewShardsPresent",
    11: "EmptyShard",
    12: "InvalidShardFlags",
    13: "InvalidIndex",
    14: "SingularMatrix",
    100: "CudaError",
    101: "AllocError",
    102: "InvalidArgument",
    103: "NoDevice",
    104: "Timeout",
    105: "LengthMismatch",
    106: "TooLarge",
}


class RsError(Exception):
    """A nonzero status from the library; `.name` is the reference Error variant."""

    def __init__(self, code):
        self.code = code
        self.name = ERROR_NAMES.get(code, "Unknown")
        msg = _lib.load().rs_strerror(code).decode()
        super().__init__("%s: %s" % (self.name, msg))


def _check(code):
    if code:
        raise RsError(code)


def _as_u8(buf, writable):
    """A uint8 numpy view of `buf` sharing its memory."""
    if isinstance(buf, np.ndarray):
        if buf.dtype != np.uint8 or not buf.flags["C_CONTIGUOUS"]:
            raise TypeError("shards must be C-contiguous uint8 arrays")
        if writable and not buf.flags["WRITEABLE"]:
            raise TypeError("output shard is read-only")
        return buf
    arr = np.frombuffer(buf, dtype=np.uint8)
    if writable and not arr.flags["WRITEABLE"]:
        raise TypeError("output shard is read-only")
    return arr


def _ptr_array(arrays):
    arr = (ctypes.c_void_p * max(len(arrays), 1))()
    for i, a in enumerate(arrays):
        arr[i] = a.ctypes.data if a.size else 0
    return arr


def _dev_ptr(x):
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _dev_ptr_array(xs):
    arr = (ctypes.c_void_p * max(len(xs), 1))()
    for i, x in enumerate(xs):
        arr[i] = _dev_ptr(x)
    return arr


def _flags(present):
    f = np.ascontiguousarray(np.asarray([bool(p) for p in present], dtype=np.uint8))
    return f, f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _same_len(arrays):
    n = len(arrays[0]) if arrays else 0
    return n, any(len(a) != n for a in arrays)


class _Coder:
    _p = ""  # "rs8" or "rs16"

    def __init__(self, data_shards, parity_shards, _handle=None):
        L = _lib.load()
        self._L = L
        if _handle is not None:
            self._h = _handle
        else:
            h = ctypes.c_void_p()
            _check(getattr(L, self._p + "_new")(data_shards, parity_shards, ctypes.byref(h)))
            self._h = h
        self._k = getattr(L, self._p + "_data_shard_count")(self._h)
        self._m = getattr(L, self._p + "_parity_shard_count")(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            getattr(self._L, self._p + "_free")(h)
            self._h = None

    def data_shard_count(self):
        return self._k

    def parity_shard_count(self):
        return self._m

    def total_shard_count(self):
        return self._k + self._m

    def clone(self):
        h = ctypes.c_void_p()
        _check(getattr(self._L, self._p + "_clone")(self._h, ctypes.byref(h)))
        return type(self)(0, 0, _handle=h)

    def __eq__(self, other):
        return type(self) is type(other) and bool(getattr(self._L, self._p + "_equal")(self._h, other._h))

    def __hash__(self):
        return hash((self._p, self._k, self._m))

    # src/reedsolomon.rs:271-278
    def encode(self, shards):
        arrs = [_as_u8(s, i >= self._k) for i, s in enumerate(shards)]
        n, uneven = _same_len(arrs)
        if len(arrs) == self.total_shard_count() and uneven:
            raise RsError(9)
        if len(arrs) == self.total_shard_count() and n == 0:
            raise RsError(11)
        _check(getattr(self._L, self._p + "_encode")(self._h, _ptr_array(arrs), len(arrs), n))

    # src/reedsolomon.rs:284-309
    def encode_sep(self, data, parity):
        d = [_as_u8(s, False) for s in data]
        p = [_as_u8(s, True) for s in parity]
        if len(d) == self._k and len(p) == self._m:
            n, uneven = _same_len(d + p)
            if uneven:
                raise RsError(9)
        else:
            n = len(d[0]) if d else 0
        _check(getattr(self._L, self._p + "_encode_sep")(
            self._h, _ptr_array(d), len(d), _ptr_array(p), len(p), n))

    # src/reedsolomon.rs:430-463
    def verify(self, shards):
        arrs = [_as_u8(s, False) for s in shards]
        n, uneven = _same_len(arrs)
        if len(arrs) == self.total_shard_count():
            if uneven:
                raise RsError(9)
            if n == 0:
                raise RsError(11)
        ok = ctypes.c_int(0)
        _check(getattr(self._L, self._p + "_verify")(self._h, _ptr_array(arrs), len(arrs), n, ctypes.byref(ok)))
        return bool(ok.value)

    def _gather(self, shards, data_only):
        """Buffers, lengths and presence of `(buf, present)` / `None` shards. `None`
        entries are allocated (zeroed) once the shard length is known, as the
        reference's Option<T> shards are (src/reedsolomon.rs:88-101)."""
        n = len(shards)
        present, lens, bufs, options = [], [], [], []
        shard_len = None
        for s in shards:
            if s is None:
                present.append(False)
                bufs.append(None)
                options.append(True)
                continue
            if isinstance(s, tuple):
                buf, p = s
            else:
                buf, p = s, True
            arr = _as_u8(buf, True)
            present.append(bool(p))
            bufs.append(arr)
            options.append(False)
            if p and shard_len is None and len(arr):
                shard_len = len(arr)
        for i in range(n):
            if options[i]:
                write = not (data_only and i >= self._k)
                bufs[i] = np.zeros(shard_len if (shard_len and write) else 0, np.uint8)
        lens = [len(b) for b in bufs]
        return bufs, lens, present, options

    def _reconstruct(self, fn, handle, shards, data_only):
        bufs, lens, present, options = self._gather(shards, data_only)
        lens_arr = (ctypes.c_size_t * max(len(lens), 1))(*lens)
        f, fp = _flags(present)
        _check(fn(handle, _ptr_array(bufs), lens_arr, fp, len(bufs), int(data_only)))
        for i, opt in enumerate(options):
            if opt and len(bufs[i]):
                shards[i] = bufs[i]

    # src/reedsolomon.rs:470-477
    def reconstruct(self, shards):
        self._reconstruct(getattr(self._L, self._p + "_reconstruct"), self._h, shards, False)

    def reconstruct_data(self, shards):
        self._reconstruct(getattr(self._L, self._p + "_reconstruct"), self._h, shards, True)

    # src/reedsolomon.rs:514-535
    def reconstruct_rows(self, rows, row_len, present):
        arr = _as_u8(rows, True)
        f, fp = _flags(present)
        _check(getattr(self._L, self._p + "_reconstruct_rows")(
            self._h, arr.ctypes.data if arr.size else None, len(arr), row_len, fp, len(f)))

    # src/reedsolomon.rs:484-505
    def prepare_decode(self, present):
        f, fp = _flags(present)
        h = ctypes.c_void_p()
        _check(getattr(self._L, self._p + "_prepare_decode")(self._h, fp, len(f), ctypes.byref(h)))
        return (PreparedDecoder if self._p == "rs8" else PreparedDecoder16)(self, h)

    # ---- device-resident variants ----
    def encode_dev(self, shards, stream=0):
        ptrs = _dev_ptr_array(shards)
        n = shards[0].numel() if hasattr(shards[0], "numel") else None
        _check(getattr(self._L, self._p + "_encode_dev")(self._h, ptrs, len(shards), n, stream))

    def encode_batch_dev(self, data, parity, row_len, n_stripes, data_stride=None, parity_stride=None,
                         stream=0):
        """Stripe s: k rows at data + s*data_stride, m rows at parity + s*parity_stride."""
        ds = data_stride if data_stride is not None else self._k * row_len
        ps = parity_stride if parity_stride is not None else self._m * row_len
        _check(getattr(self._L, self._p + "_encode_batch_dev")(
            self._h, _dev_ptr(data), ds, _dev_ptr(parity), ps, n_stripes, row_len, stream))

    def reconstruct_dev(self, shards, present, shard_len, data_only=False, stream=0):
        ptrs = _dev_ptr_array(shards)
        lens = (ctypes.c_size_t * len(shards))(*([shard_len] * len(shards)))
        f, fp = _flags(present)
        _check(getattr(self._L, self._p + "_reconstruct_dev")(
            self._h, ptrs, lens, fp, len(shards), int(data_only), stream))

    # ---- payload framing (rs*_frame_*: the callers' steps either side of the coder) ----
    def frame_encode_dev(self, payload, shard_len, stream=0):
        """payload: 1-D uint8 CUDA tensor -> stripes (S, n, shard_len) on the device: the
        payload's bytes fill the data shards in order (zeros after it), parity encoded."""
        import torch

        length = payload.numel()
        S = frame_stripe_count(length, self._k, shard_len)
        stripes = torch.empty((S, self._k + self._m, shard_len), dtype=torch.uint8, device=payload.device)
        _check(getattr(self._L, self._p + "_frame_encode_dev")(
            self._h, _dev_ptr(payload) if length else None, length, shard_len,
            _dev_ptr(stripes) if S else None, S, stream))
        return stripes

    def frame_decode_dev(self, stripes, shard_len, present, payload_len, stream=0):
        """Rebuild every stripe's missing data shards (present: (S, n) flags) and
        reassemble the payload. Returns (payload tensor, per-stripe statuses): a stripe
        with too few shards reports its error there (its payload bytes are not rebuilt);
        argument and device errors raise."""
        import torch

        S = stripes.shape[0] if stripes.dim() else 0
        f = np.ascontiguousarray(np.asarray(present, dtype=np.uint8).reshape(S, self._k + self._m))
        out = torch.empty(payload_len, dtype=torch.uint8, device=stripes.device)
        st = (ctypes.c_int * max(S, 1))()
        code = getattr(self._L, self._p + "_frame_decode_dev")(
            self._h, _dev_ptr(stripes) if S else None, S, shard_len,
            f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), _dev_ptr(out) if payload_len else None,
            payload_len, st, stream)
        if code >= 100 or code in (9, 11):
            _check(code)
        return out, list(st)[:S]


def frame_stripe_count(payload_len, data_shards, shard_len):
    """Stripes a payload fills at k data shards of shard_len bytes each."""
    return _lib.load().rs_frame_stripe_count(payload_len, data_shards, shard_len)


def outer_shape(groups):
    """The tape outer coder's (k, m) for `groups` groups: k = ceil(groups / 3)."""
    k, m = ctypes.c_size_t(0), ctypes.c_size_t(0)
    _check(_lib.load().rs_outer_shape(groups, ctypes.byref(k), ctypes.byref(m)))
    return k.value, m.value


def outer_shard_bytes(segment_len, data_shards):
    """The outer coder's shard size: ceil(segment / k) rounded up to 64, at most 4 MiB."""
    s = ctypes.c_size_t(0)
    _check(_lib.load().rs_outer_shard_bytes(segment_len, data_shards, ctypes.byref(s)))
    return s.value


class ReedSolomon(_Coder):
    """ReedSolomon over GF(2^8), src/reedsolomon.rs:139-196."""

    _p = "rs8"

    def parity_matrix(self):
        out = np.zeros(self._m * self._k, np.uint8)
        _check(self._L.rs8_parity_matrix(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), out.size))
        return out.reshape(self._m, self._k)

    def encode_route(self, shard_len):
        return self._L.rs8_encode_route(self._h, shard_len).decode()

    def set_route(self, route):
        """0 = automatic, 1 = matrix kernel, 2 = the shape's compiled bitsliced kernel (FFT or
        generator) where one exists."""
        _check(self._L.rs8_set_route(self._h, {"auto": 0, "matrix": 1, "fft": 2}.get(route, route)))

    def encode_fused(self, shards):
        """Alias of encode, src/reedsolomon.rs:354-359."""
        self.encode(shards)

    # src/reedsolomon.rs:652-697
    def encode_rows(self, data, row_len):
        d = _as_u8(data, False)
        if len(d) != self._k * row_len:
            raise AssertionError("data must be data_shard_count * row_len bytes")
        parity = np.zeros(self._m * row_len, np.uint8)
        self.encode_rows_into(d, row_len, parity)
        return parity

    def encode_rows_into(self, data, row_len, parity):
        d = _as_u8(data, False)
        p = _as_u8(parity, True)
        _check(self._L.rs8_encode_rows(self._h, d.ctypes.data if d.size else None, len(d), row_len,
                                       p.ctypes.data if p.size else None, len(p)))

    def encode_batch_host(self, data, parity, row_len, n_stripes, data_stride=None, parity_stride=None):
        """Stripes from host memory (numpy arrays; pinned memory copies fastest)."""
        d = _as_u8(data.reshape(-1) if isinstance(data, np.ndarray) else data, False)
        p = _as_u8(parity.reshape(-1) if isinstance(parity, np.ndarray) else parity, True)
        ds = data_stride if data_stride is not None else self._k * row_len
        ps = parity_stride if parity_stride is not None else self._m * row_len
        if len(d) < ds * (n_stripes - 1) + self._k * row_len or len(p) < ps * (n_stripes - 1) + self._m * row_len:
            raise RsError(9)
        _check(self._L.rs8_encode_batch(self._h, d.ctypes.data, ds, p.ctypes.data, ps, n_stripes, row_len))

    def encode_rows_dev(self, data, row_len, parity, stream=0):
        _check(self._L.rs8_encode_rows_dev(self._h, _dev_ptr(data), row_len, _dev_ptr(parity), stream))

    def verify_dev(self, shards, shard_len, stream=0):
        ok = ctypes.c_int(0)
        _check(self._L.rs8_verify_dev(self._h, _dev_ptr_array(shards), len(shards), shard_len,
                                      ctypes.byref(ok), stream))
        return bool(ok.value)

    def reconstruct_batch_dev(self, rows, n_stripes, row_len, present, stripe_stride=None,
                              data_only=False, stream=0):
        """present: (n_stripes, n) flags. Returns the per-stripe status list."""
        n = self.total_shard_count()
        ss = stripe_stride if stripe_stride is not None else n * row_len
        f = np.ascontiguousarray(np.asarray(present, dtype=np.uint8).reshape(n_stripes, n))
        st = (ctypes.c_int * max(n_stripes, 1))()
        _check(self._L.rs8_reconstruct_batch_dev(
            self._h, _dev_ptr(rows), ss, n_stripes, row_len, f.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            int(data_only), st, stream))
        return list(st)[:n_stripes]


class ReedSolomon16(_Coder):
    """ReedSolomon16 over GF((2^8)^2), split-plane shards, src/reedsolomon16.rs:252-319."""

    _p = "rs16"

    def parity_matrix(self):
        out = np.zeros(self._m * self._k, np.uint16)
        _check(self._L.rs16_parity_matrix(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), out.size))
        return out.reshape(self._m, self._k)

    def encode_route(self, shard_len=None, n_stripes=1):
        """The shape's route ("fft", "matrix", or "subfield" when k + m <= 256 and the
        GF(2^8) codec of the shape does the work), or with shard_len the route of an
        encode of n_stripes stripes of that shard length."""
        if shard_len is None:
            return self._L.rs16_encode_route(self._h).decode()
        return self._L.rs16_encode_route_for(self._h, shard_len, n_stripes).decode()

    def set_route(self, route):
        """Test hook: "auto", "matrix" or "fft" (identical bytes on every route)."""
        _check(self._L.rs16_set_route(self._h, {"auto": 0, "matrix": 1, "fft": 2}[route]))

    def encode(self, shards):
        arrs = [_as_u8(s, i >= self._k) for i, s in enumerate(shards)]
        if len(arrs) == self.total_shard_count():
            n = None
            for a in arrs:  # note_shard_len order, src/reedsolomon16.rs:758-772
                if len(a) == 0:
                    raise RsError(11)
                if len(a) % 2:
                    raise RsError(9)
                if n is not None and n != len(a):
                    raise RsError(9)
                n = len(a)
        super().encode(arrs)

    def encode_sep(self, data, parity):
        d = [_as_u8(s, False) for s in data]
        p = [_as_u8(s, True) for s in parity]
        if len(d) == self._k and len(p) == self._m:
            n = None
            for a in d + p:
                if len(a) == 0:
                    raise RsError(11)
                if len(a) % 2:
                    raise RsError(9)
                if n is not None and n != len(a):
                    raise RsError(9)
                n = len(a)
        super().encode_sep(d, p)


class _Prepared:
    _fn = ""

    def __init__(self, coder, handle):
        self._coder = coder
        self._L = coder._L
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            getattr(self._L, self._fn + "_dec_free")(h)
            self._h = None

    def reconstruct(self, shards):
        self._coder._reconstruct(getattr(self._L, self._fn + "_dec_reconstruct"), self._h, shards, False)

    def reconstruct_data(self, shards):
        self._coder._reconstruct(getattr(self._L, self._fn + "_dec_reconstruct"), self._h, shards, True)

    def clone(self):
        h = ctypes.c_void_p()
        _check(getattr(self._L, self._fn + "_dec_clone")(self._h, ctypes.byref(h)))
        return type(self)(self._coder, h)


class PreparedDecoder(_Prepared):
    """PreparedDecoder, src/reedsolomon.rs:749-797."""

    _fn = "rs8"


class PreparedDecoder16(_Prepared):
    """PreparedDecoder16, src/reedsolomon16.rs:705-753."""

    _fn = "rs16"


class _BatchItem(ctypes.Structure):
    _fields_ = [("codec", ctypes.c_void_p), ("d_rows", ctypes.c_void_p), ("row_stride", ctypes.c_size_t),
                ("row_len", ctypes.c_size_t), ("op", ctypes.c_int), ("present", ctypes.POINTER(ctypes.c_uint8))]


ENCODE, RECONSTRUCT, RECONSTRUCT_DATA = 0, 1, 2
MATRIX_ONLY, NO_GRAPH = 1, 2


def _batch_items(items):
    """rs_batch_item array for (codec, rows, row_stride, row_len, op, present) tuples, and
    the flag arrays it points into (keep them alive while it is used)."""
    arr = (_BatchItem * max(len(items), 1))()
    keep = []
    for i, (codec, rows, stride, row_len, op, present) in enumerate(items):
        arr[i].codec = codec._h.value
        arr[i].d_rows = _dev_ptr(rows)
        arr[i].row_stride = stride
        arr[i].row_len = row_len
        arr[i].op = op
        if present is not None:
            f, fp = _flags(present)
            keep.append(f)
            arr[i].present = fp
    return arr, keep


class Queue:
    """Persistent work queue (rs_queue_*): start() launches one persistent kernel; push()
    hands it stripes (the Batch item tuples) while it runs; finish() closes the session
    and returns its status (0, or the Timeout code 104 when a device wait gave up);
    wait() waits without closing. Rows must stay valid until the session ends. While a
    session runs, free no device or pinned memory (destroying a codec does): CUDA's
    frees synchronize the device and would wait for the session's kernel, which ends
    only at close or at its timeout. start() collects garbage first for that reason."""

    def __init__(self, max_units=1 << 16, arena_bytes=0, timeout_s=1.0):
        self._L = _lib.load()
        h = ctypes.c_void_p()
        _check(self._L.rs_queue_create(max_units, arena_bytes, int(timeout_s * 1e9), ctypes.byref(h)))
        self._h = h
        self._hold = []

    def start(self):
        import gc

        self._hold = []
        gc.collect()  # pending codec frees would otherwise wait for the session's kernel
        _check(self._L.rs_queue_start(self._h))

    def push(self, items):
        arr, keep = _batch_items(items)
        st = (ctypes.c_int * max(len(items), 1))()
        _check(self._L.rs_queue_push(self._h, arr, len(items), st))
        self._hold.append((items, keep))
        return list(st)[:len(items)]

    def progress(self):
        d, p = ctypes.c_uint64(), ctypes.c_uint64()
        _check(self._L.rs_queue_progress(self._h, ctypes.byref(d), ctypes.byref(p)))
        return d.value, p.value

    def _end(self, fn):
        code = fn(self._h)
        if code not in (0, 104):
            _check(code)
        return code

    def finish(self):
        return self._end(self._L.rs_queue_finish)

    def wait(self):
        return self._end(self._L.rs_queue_wait)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.rs_queue_free(h)
            self._h = None


class Batch:
    """A mixed batch of GF(2^8) stripes (rs_batch_create): items are tuples
    (codec, rows, row_stride, row_len, op, present) with `rows` a CUDA tensor or device
    pointer holding n = k+m rows; `present` (n flags) for reconstruct ops.

    Launch configurations: `configs` gives one per item (an index into
    tuner.CONFIGS, -1 automatic; rs_batch_create_configured); `model` (a
    tuner.CostModel, e.g. tuner.shipped_model()) lets the cost model choose them
    (rs_batch_choose). Neither changes the bytes."""

    def __init__(self, items, flags=0, configs=None, model=None):
        self._L = _lib.load()
        n = len(items)
        arr, self._keep = _batch_items(items)
        self._codecs = [it[0] for it in items]
        st = (ctypes.c_int * max(n, 1))()
        h = ctypes.c_void_p()
        if model is not None:
            cfg = (ctypes.c_int * max(n, 1))()
            _check(self._L.rs_batch_choose(arr, n, model._h, cfg))
            configs = list(cfg)[:n]
        self.configs = list(configs) if configs is not None else None
        if configs is None:
            _check(self._L.rs_batch_create(arr, n, flags, st, ctypes.byref(h)))
        else:
            cfg = (ctypes.c_int * max(n, 1))(*configs)
            _check(self._L.rs_batch_create_configured(arr, n, flags, cfg, st, ctypes.byref(h)))
        self._h = h
        self.statuses = list(st)[:n]

    def launch(self, stream=0):
        _check(self._L.rs_batch_launch(self._h, stream))

    def stats(self):
        la, fi, mi = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        by = ctypes.c_uint64()
        _check(self._L.rs_batch_stats(self._h, ctypes.byref(la), ctypes.byref(fi), ctypes.byref(mi), ctypes.byref(by)))
        return {"launches": la.value, "fft_items": fi.value, "matrix_items": mi.value, "bytes": by.value}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.rs_batch_free(h)
            self._h = None


# gf::mul_slice / mul_slice_xor, src/gf/mod.rs:69-85
def mul_slice(out, inp, c):
    o = _as_u8(out, True)
    i = _as_u8(inp, False)
    _check(_lib.load().gf8_mul_slice(o.ctypes.data if o.size else None, len(o),
                                     i.ctypes.data if i.size else None, len(i), c, 0))


def mul_slice_xor(out, inp, c):
    o = _as_u8(out, True)
    i = _as_u8(inp, False)
    _check(_lib.load().gf8_mul_slice(o.ctypes.data if o.size else None, len(o),
                                     i.ctypes.data if i.size else None, len(i), c, 1))


def mul_slice_dev(out, inp, n, c, xor_into=False, stream=0):
    _check(_lib.load().gf8_mul_slice_dev(_dev_ptr(out), _dev_ptr(inp), n, c, int(xor_into), stream))


def device_check():
    return _lib.load().rs_device_check()


def kernel_launch_count():
    return _lib.load().rs_kernel_launch_count()
