"""Device-side orchestration of the imaging path: plans, band selection and the batched SOCS / Abbe calls.

Every image the reference computes has the form
    I[y, x] = sum_fields w * | sum_{m in band} P(m) c(m) exp(-2 pi i (m_r y/Ny + m_c x/Nx)) |^2
with c(m) = 1/(Ny Nx) sum h[y, x] exp(+2 pi i (m_r y/Ny + m_c x/Nx)) the mask spectrum:
  * Abbe (CalculateAerialImage.py:18-103): fields = (source point j, polarisation component e, channel),
    P = shifted pupil of point j, w = n * v_j / sum(v);
  * SOCS (CalculateAerialImage_SOCS.py:3-11): fields = (kernel k, channel), P = kernel k, w = 1.
The engine computes it in three native stages (liboi_b200):
  1. oi_band_spectrum   -- c(m) on the band only (Br x Bc frequencies), from the mask in one pass;
  2. oi_coherent_coarse -- sum of |field|^2 on a coarse Mr x Mc grid (Mr >= 2Br-1), fields kept on chip;
  3. oi_coarse_to_image -- exact band-limited resampling of that intensity to the Ny x Nx output.
Stage 3 is exact because the intensity's spectrum lives on |q| < B; the result equals the reference's full
grid FFT evaluation index for index.
"""
from __future__ import annotations

import collections
import math
import threading
from dataclasses import dataclass

import torch

from . import _native as N

COARSE_ALIGN = 64


def coarse_size(b: int) -> int:
    """Smallest multiple of 64 that holds the 2B-1 intensity frequencies of a B-wide band."""
    return max(COARSE_ALIGN, ((2 * b - 1 + COARSE_ALIGN - 1) // COARSE_ALIGN) * COARSE_ALIGN)


def require_cuda(device=None) -> torch.device:
    if not torch.cuda.is_available():
        raise N.NativeError('opticalimaging_b200 needs a CUDA device; there is no CPU path')
    d = torch.device(device) if device is not None else torch.device('cuda', torch.cuda.current_device())
    if d.type != 'cuda' or d.index is None:   # 'cuda' alone means the current device
        d = torch.device('cuda', torch.cuda.current_device())
    N.load()
    return d


def twiddle(rows, cols, a0, b0, n, sign, device, scale=1.0):
    """exp(sign 2 pi i (a+a0)(b+b0)/n) as a [rows, cols] complex64 device tensor."""
    out = torch.empty((rows, cols), dtype=torch.complex64, device=device)
    N.call('oi_twiddle', N.ptr(out), rows, cols, a0, b0, n, sign, float(scale), N.stream_handle(device))
    return out


def fft_tables(n: int, device) -> torch.Tensor:
    """Twiddle tables of the n-point four-step FFT (n = 32 n1): t2[k2][j] = exp(+2 pi i k2 j / n) (32 x n1)
    followed by t1[k1][j] = exp(+2 pi i k1 j / n1) (n1 x n1), one complex64 buffer."""
    n1 = n // 32
    return torch.cat([twiddle(32, n1, 0, 0, n, +1, device).reshape(-1),
                      twiddle(n1, n1, 0, 0, n1, +1, device).reshape(-1)])


@dataclass(frozen=True)
class Band:
    """Centred frequency band: rows m0r .. m0r+br-1, columns m0c .. m0c+bc-1."""
    m0r: int
    br: int
    m0c: int
    bc: int


FORMS = ('fft', 'dft', 'bf16x3')
TC_COARSE = (128, 128)      # the coarse grid of the tensor-core (split-BF16x3) coherent contraction


def tc_supported(band: Band) -> bool:
    """The split-BF16x3 contraction covers bands of at most 64 x 64 (coarse grid 128 x 128)."""
    return band.br <= 64 and band.bc <= 64


def fft_supported(ny: int, nx: int, band: Band) -> bool:
    """The FFT form covers power-of-two grids of 256..2048 per axis with the band inside Nyquist."""
    lib = N.load()
    if not lib.oi_fft_supported(ny, nx):
        return False
    maxc = max(abs(band.m0c), abs(band.m0c + band.bc - 1))
    return 2 * maxc < nx and band.br <= ny and 2 * band.br - 1 <= ny and 2 * band.bc - 1 <= nx


class Plan:
    """Phase tables for one (output grid, band); cached and shared by every call with the same key.  The cache
    keeps the CACHE_SIZE most recently used plans (a model holds on to its own plan regardless)."""

    CACHE_SIZE = 64
    _cache: collections.OrderedDict = collections.OrderedDict()
    _lock = threading.Lock()

    def __init__(self, ny, nx, band: Band, device, coarse=None):
        self.ny, self.nx, self.band, self.device = ny, nx, band, device
        b = band
        self.mr, self.mc = coarse if coarse is not None else (coarse_size(b.br), coarse_size(b.bc))
        if self.mr < 2 * b.br - 1 or self.mc < 2 * b.bc - 1 or self.mc % 64:
            raise ValueError(f'coarse grid {self.mr}x{self.mc} cannot hold the intensity of band {b.br}x{b.bc}')
        nq = 2 * b.br - 1
        t = lambda *a: twiddle(*a, device=device)  # noqa: E731
        self.wx = t(nx, b.bc, 0, b.m0c, nx, +1)              # [nx][bc]   forward x
        self.wy = t(ny, b.br, 0, b.m0r, ny, +1)              # [ny][br]   forward y
        self.frow = t(self.mr, b.br, 0, b.m0r, self.mr, -1)  # [mr][br]   coarse rows
        self.fcol = t(b.bc, self.mc, b.m0c, 0, self.mc, -1)  # [bc][mc]   coarse columns
        self.gc = t(self.mc, b.bc, 0, 0, self.mc, +1)        # [mc][bc]   coarse -> spectrum (x)
        self.gr = t(self.mr, nq, 0, -(b.br - 1), self.mr, +1)  # [mr][2br-1]
        self.sy = t(ny, nq, 0, -(b.br - 1), ny, -1)          # [ny][2br-1] spectrum -> image (y)
        self.sx = t(b.bc, nx, 0, 0, nx, -1)                  # [bc][nx]   spectrum -> image (x)
        self.fft = fft_supported(ny, nx, band)
        if self.fft:                                          # the FFT form's twiddle tables per axis
            self.wn_x = fft_tables(nx, device)
            self.wn_y = fft_tables(ny, device)
        self.coarse_fft = self.mr in (64, 128) and self.mc in (64, 128)
        self.coarse256 = (self.mr, self.mc) == (256, 256)     # the tensor-memory accumulator kernel
        if self.coarse_fft or self.coarse256:                 # the coarse-grid FFT tables
            self.wm_r = t(1, self.mr, 1, 0, self.mr, +1)
            self.wm_c = t(1, self.mc, 1, 0, self.mc, +1)

    def tc_constants(self) -> torch.Tensor:
        """The split DFT operand image of the tensor-core form (built once per plan; coarse grid 128 x 128)."""
        c = getattr(self, '_tc_consts', None)
        if c is None:
            b = self.band
            nbytes = 98304 if b.m0r == b.m0c else 163840
            c = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            N.call('oi_tc_constants', b.m0r, b.m0c, N.ptr(self.wm_r), N.ptr(self.wm_c), N.ptr(c), nbytes,
                   N.stream_handle(self.device))
            self._tc_consts = c
        return c

    def tc_rows(self, form) -> bool:
        """The split-BF16x3 form runs the N-point row passes on the tensor cores too (FFT grids, band <= 64)."""
        b = self.band
        return (form == 'bf16x3' and self.fft and self.ny % 128 == 0 and self.nx % 128 == 0 and b.bc <= 64
                and b.br <= 64)

    def symmetric_band(self) -> bool:
        """Odd band centred on frequency 0 in both axes (m0 = -(b-1)/2): a real mask's band spectrum then follows
        from its non-negative columns, band[-ky][-kx] = conj(band[ky][kx])."""
        b = self.band
        return b.br % 2 == 1 and b.bc % 2 == 1 and b.m0r == -(b.br - 1) // 2 and b.m0c == -(b.bc - 1) // 2

    def rows_consts(self, which: int) -> torch.Tensor:
        """Constant operand image of the tensor-core row pass: 0 forward (band columns), 1 inverse (synthesis),
        2 forward over the non-negative half of a symmetric band."""
        attr = '_rows_consts_%d' % which
        c = getattr(self, attr, None)
        if c is None:
            b = self.band
            nbytes = {0: (self.nx // 64) * 32768, 1: (self.nx // 128) * 65536, 2: (self.nx // 64) * 16384}[which]
            c = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            N.call('oi_rows_tc_constants', which, self.nx, b.m0c, b.bc, N.ptr(c), nbytes, N.stream_handle(self.device))
            setattr(self, attr, c)
        return c

    def synth_consts(self) -> torch.Tensor:
        """Constant operands of the tensor-core synthesis preparation (oi_synth_tc_constants: the coarse spectrum's
        column DFT and the row Dirichlet kernels of this grid and band), built once per plan."""
        c = getattr(self, '_synth_consts', None)
        if c is None:
            b = self.band
            nbytes = (1 + self.ny // 128) * 65536
            c = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            N.call('oi_synth_tc_constants', self.ny, b.br, b.bc, N.ptr(c), nbytes, N.stream_handle(self.device))
            self._synth_consts = c
        return c

    def coarse_fft_tables(self):
        """Four-step FFT tables of the coarse grid (for coarse grids of 256..2048 points per axis)."""
        t = getattr(self, '_coarse_fft_tables', None)
        if t is None:
            t = self._coarse_fft_tables = (fft_tables(self.mr, self.device), fft_tables(self.mc, self.device))
        return t

    def big_coarse_fft(self, form) -> bool:
        """Coarse grids above 128 (bands over 64) on FFT output grids: the coarse spectrum by the FFT band pass."""
        lib = N.load()
        return (form != 'dft' and self.fft and not self.coarse_fft and lib.oi_fft_supported(self.mr, self.mc) == 1
                and 2 * (self.band.bc - 1) < self.mc and 2 * self.band.br - 1 <= self.mr)

    def use_fft(self, form):
        if form not in (None,) + FORMS:
            raise ValueError(f'form must be one of {FORMS}')
        return self.fft and form != 'dft'

    def use_coarse_fft(self, form):
        return self.coarse_fft and form != 'dft'

    def use_coarse256(self, form):
        return self.coarse256 and form != 'dft'


    @classmethod
    def get(cls, ny, nx, band: Band, device, coarse=None) -> 'Plan':
        key = (ny, nx, band, str(device), coarse)
        with cls._lock:
            p = cls._cache.get(key)
            if p is None:
                p = cls._cache[key] = cls(ny, nx, band, device, coarse)
                while len(cls._cache) > cls.CACHE_SIZE:
                    cls._cache.popitem(last=False)
            else:
                cls._cache.move_to_end(key)
            return p


B200_SMS = 148          # the SM count assumed for host-side layout arithmetic when no device is visible
_SM_COUNTS: dict = {}


def sm_count() -> int:
    """Streaming multiprocessors of the current device (148 on a B200): the grids of the one-block-per-SM
    kernels and the field splits below are sized by it, as the native layouts are."""
    if not torch.cuda.is_available():
        return B200_SMS
    d = torch.cuda.current_device()
    n = _SM_COUNTS.get(d)
    if n is None:
        n = _SM_COUNTS[d] = torch.cuda.get_device_properties(d).multi_processor_count
    return n


def tc_parts_bound(images: int, fields: int, ctas: int | None = None) -> int:
    """Upper bound of the partial-sum slots oi_coherent_coarse_tc needs (for workspace estimates)."""
    tasks = images * fields
    g = min(sm_count() if ctas is None else ctas, tasks)
    return min(fields, -(-fields * g // tasks) + 1)


def field_split(nfields: int, blocks: int, sms: int | None = None) -> int:
    """Smallest divisor d of nfields with blocks * d >= 3 waves of one block per SM (nfields if none)."""
    target = 3 * (sm_count() if sms is None else sms)
    for d in range(1, nfields + 1):
        if nfields % d == 0 and blocks * d >= target:
            return d
    return nfields


def field_split_sm(nfields: int, blocks: int, sms: int | None = None) -> int:
    """Field split for a kernel of one block per SM (the 256 x 256 coarse grid): the d minimising
    waves(d) * (fields per block + 1/2), the half standing for a block's fixed start and partial-sum write;
    ties go to the smaller d (fewer partial sums)."""
    sms = sm_count() if sms is None else sms
    best, best_cost = 1, None
    for d in range(1, nfields + 1):
        cost = -(-blocks * d // sms) * (-(-nfields // d) + 0.5)
        if best_cost is None or cost < best_cost:
            best, best_cost = d, cost
    return best


# --------------------------------------------------------------------------------------------- stages
def band_spectrum(field: torch.Tensor, kind: int, plan: Plan, nch: int = 1, scale: float = 1.0,
                  scratch: torch.Tensor | None = None, form: str | None = None) -> torch.Tensor:
    """c(m) on the plan's band: [batch, nch, br, bc] complex64.

    field: float32 [B, ny, nx] (FIELD_REAL_F32), uint8 [B, ny, nx] (FIELD_U8) or complex64 [B, ny, nx, nch]
    (FIELD_COMPLEX_C64), contiguous on the plan's device.  `scale` multiplies the 1/(ny nx) normalisation.
    form: 'fft' (default where the grid allows: real or uint8 masks on 256..2048 power-of-two grids) or 'dft'.
    """
    b = plan.band
    batch = field.shape[0]
    need = batch * nch * plan.ny * b.bc
    if scratch is None or scratch.numel() < need:
        scratch = torch.empty(need, dtype=torch.complex64, device=plan.device)
    band = torch.empty((batch, nch, b.br, b.bc), dtype=torch.complex64, device=plan.device)
    s = N.stream_handle(plan.device)
    sc = float(scale / (plan.ny * plan.nx))
    if plan.tc_rows(form) and kind != N.FIELD_COMPLEX_C64 and nch == 1 and plan.symmetric_band():
        N.call('oi_band_spectrum_tc_sym', N.ptr(field), kind, batch, plan.ny, plan.nx, b.br, b.bc,
               N.ptr(plan.rows_consts(2)), N.ptr(plan.wn_y), sc, N.ptr(scratch), N.ptr(band), s)
    elif plan.tc_rows(form) and kind != N.FIELD_COMPLEX_C64 and nch == 1:
        N.call('oi_band_spectrum_tc', N.ptr(field), kind, batch, plan.ny, plan.nx, b.m0r, b.br, b.m0c, b.bc,
               N.ptr(plan.rows_consts(0)), N.ptr(plan.wn_y), sc, N.ptr(scratch), N.ptr(band), s)
    elif plan.use_fft(form) and kind != N.FIELD_COMPLEX_C64 and nch == 1:
        N.call('oi_band_spectrum_fft', N.ptr(field), kind, batch, plan.ny, plan.nx, b.m0r, b.br, b.m0c, b.bc,
               N.ptr(plan.wn_x), N.ptr(plan.wn_y), sc, N.ptr(scratch), N.ptr(band), s)
    else:
        N.call('oi_band_spectrum', N.ptr(field), kind, batch, plan.ny, plan.nx, nch, b.br, b.bc, N.ptr(plan.wx),
               N.ptr(plan.wy), sc, N.ptr(scratch), N.ptr(band), s)
    return band


def _mark(marks, name):
    if marks is not None:
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        marks.append((name, ev))


def coherent_image(band: torch.Tensor, pupils: torch.Tensor, weights: torch.Tensor, plan: Plan,
                   pupil_batch_stride: int = 0, out: torch.Tensor | None = None, marks=None,
                   form: str | None = None) -> torch.Tensor:
    """sum_fields w |IDFT(P .* c)|^2 on the output grid: [batch, nz, ny, nx] float32.

    band: [batch, nch, br, bc] complex64; pupils: [nz, nk, br, bc] complex64 (shared by the batch when
    pupil_batch_stride == 0); weights: [nz, nk] float32.
    """
    b = plan.band
    batch, nch = band.shape[0], band.shape[1]
    nz, nk = pupils.shape[-4], pupils.shape[-3]
    dev = plan.device
    s = N.stream_handle(dev)
    if form == 'bf16x3':
        if not tc_supported(b):
            raise ValueError(f'the bf16x3 form covers bands up to 64 x 64 (this one is {b.br} x {b.bc})')
        if (plan.mr, plan.mc) != TC_COARSE:
            plan = Plan.get(plan.ny, plan.nx, b, dev, coarse=TC_COARSE)
        ctas, nsplit = N.tc_layout(batch * nz, nk * nch)
        coarse = torch.empty((nsplit, batch, nz, plan.mr, plan.mc), dtype=torch.float32, device=dev)
        N.call('oi_coherent_coarse_tc', N.ptr(band), batch, nch, b.m0r, b.br, b.m0c, b.bc, N.ptr(pupils),
               int(pupil_batch_stride), N.ptr(weights), nz, nk, N.ptr(plan.tc_constants()), ctas, nsplit,
               N.ptr(coarse), s)
    elif plan.use_coarse_fft(form) or plan.use_coarse256(form):
        nsplit = (field_split_sm(nk * nch, batch * nz) if plan.coarse256 else field_split(nk * nch, batch * nz))
        coarse = torch.empty((nsplit, batch, nz, plan.mr, plan.mc), dtype=torch.float32, device=dev)
        N.call('oi_coherent_coarse_fft', N.ptr(band), batch, nch, b.m0r, b.br, b.m0c, b.bc, N.ptr(pupils),
               int(pupil_batch_stride), N.ptr(weights), nz, nk, plan.mr, plan.mc, N.ptr(plan.wm_r),
               N.ptr(plan.wm_c), nsplit, N.ptr(coarse), s)
    else:
        nsplit = field_split(nk * nch, batch * nz * ((plan.mr + 15) // 16))
        coarse = torch.empty((nsplit, batch, nz, plan.mr, plan.mc), dtype=torch.float32, device=dev)
        N.call('oi_coherent_coarse', N.ptr(band), batch, nch, b.br, b.bc, N.ptr(pupils), int(pupil_batch_stride),
               N.ptr(weights), nz, nk, plan.mr, plan.mc, N.ptr(plan.frow), N.ptr(plan.fcol), nsplit, N.ptr(coarse),
               s)
    _mark(marks, 'coherent_coarse')
    if out is None:
        out = torch.empty((batch, nz, plan.ny, plan.nx), dtype=torch.float32, device=dev)
    ihat = torch.empty(batch * nz * (2 * b.br - 1) * b.bc, dtype=torch.complex64, device=dev)
    if form == 'bf16x3' and plan.tc_rows(form):
        # coarse spectrum and column synthesis as two tensor-core GEMMs straight into the row pass's operand tiles
        tiles = torch.empty(batch * nz * plan.ny * 512, dtype=torch.uint8, device=dev)
        N.call('oi_coarse_to_image_tcs', N.ptr(coarse), nsplit, batch * nz, b.br, b.bc, N.ptr(plan.synth_consts()),
               N.ptr(plan.rows_consts(1)), plan.ny, plan.nx, N.ptr(tiles), N.ptr(out), s)
    elif plan.big_coarse_fft(form):
        # the coarse intensity's Hermitian half-spectrum by the FFT band pass, then the FFT synthesis
        count = batch * nz
        wn_r, wn_c = plan.coarse_fft_tables()
        t = torch.empty(count * plan.mr * b.bc, dtype=torch.complex64, device=dev)
        N.call('oi_coarse_half_spectrum_fft', N.ptr(coarse), nsplit, count, plan.mr, plan.mc, b.br, b.bc, N.ptr(wn_c),
               N.ptr(wn_r), N.ptr(t), N.ptr(ihat), s)
        v = torch.empty(count * b.bc * plan.ny, dtype=torch.complex64, device=dev)
        N.call('oi_spectrum_to_image_fft', N.ptr(ihat), count, b.br, b.bc, N.ptr(plan.wn_y), N.ptr(plan.wn_x),
               plan.ny, plan.nx, N.ptr(v), N.ptr(out), s)
    elif plan.use_fft(form):
        v = torch.empty(batch * nz * b.bc * plan.ny, dtype=torch.complex64, device=dev)
        wm_r, wm_c = (plan.wm_r, plan.wm_c) if plan.coarse_fft else (None, None)
        N.call('oi_coarse_to_image_fft', N.ptr(coarse), nsplit, batch * nz, plan.mr, plan.mc, b.br, b.bc,
               N.ptr(plan.gc), N.ptr(plan.gr), N.ptr(wm_r), N.ptr(wm_c), N.ptr(plan.wn_y), N.ptr(plan.wn_x),
               plan.ny, plan.nx, N.ptr(ihat), N.ptr(v), N.ptr(out), s)
    else:
        N.call('oi_coarse_to_image', N.ptr(coarse), nsplit, batch * nz, plan.mr, plan.mc, b.br, b.bc,
               N.ptr(plan.gc), N.ptr(plan.gr), N.ptr(plan.sy), N.ptr(plan.sx), plan.ny, plan.nx, N.ptr(ihat),
               N.ptr(out), s)
    _mark(marks, 'coarse_to_image')
    return out


# --------------------------------------------------------------------------------------------- bands
def clip_band(lo: int, hi: int, n: int):
    """Intersect the centred frequency interval [lo, hi] with the grid's frequencies [-(n//2), (n+1)//2 - 1]."""
    lo = max(lo, -(n // 2))
    hi = min(hi, (n + 1) // 2 - 1)
    return lo, hi


def abbe_band(ny, nx, npy, npx, sx: torch.Tensor, sy: torch.Tensor) -> Band | None:
    """Band covering every shifted pupil |m_r/npy + X|^2 + |m_c/npx + Y|^2 <= 1 (rows carry the source X,
    CalculateAerialImage.py:31,55), widened by one frequency for float32 rounding; None if empty."""
    xmax, xmin = float(sx.max()), float(sx.min())
    ymax, ymin = float(sy.max()), float(sy.min())
    r0, r1 = clip_band(math.floor(npy * (-1 - xmax)) - 1, math.ceil(npy * (1 - xmin)) + 1, ny)
    c0, c1 = clip_band(math.floor(npx * (-1 - ymax)) - 1, math.ceil(npx * (1 - ymin)) + 1, nx)
    if r1 < r0 or c1 < c0:
        return None
    return Band(r0, r1 - r0 + 1, c0, c1 - c0 + 1)


def cyclic_support(nonzero: torch.Tensor):
    """Smallest cyclic interval [start, start+length) of indices covering every True entry."""
    n = nonzero.numel()
    idx = torch.nonzero(nonzero).flatten().tolist()
    if not idx:
        return 0, 1
    if len(idx) == 1:
        return idx[0], 1
    gaps = [(idx[(i + 1) % len(idx)] - idx[i]) % n for i in range(len(idx))]
    i = max(range(len(idx)), key=lambda k: gaps[k])
    if gaps[i] <= 1:
        return 0, n
    start = idx[(i + 1) % len(idx)]
    return start, n - gaps[i] + 1


def centred(start: int, n: int) -> int:
    """Representative of index `start` (mod n) in the centred range [-(n//2), n - n//2)."""
    s = start % n
    return s - n if s >= n - n // 2 else s


# ------------------------------------------------------------------------------------- resident models
def pack_real_fields(pupils: torch.Tensor, weights: torch.Tensor, band: Band, tol: float = 1e-14):
    """The fields of a model, packed two to a transform for real masks.

    A real mask's band spectrum c is Hermitian on a band centred on frequency 0: c(-f) = conj c(f).  So is the
    product of two Hermitian arrays, and a Hermitian spectrum transforms to a real field.  A weighted field
    Q = sqrt(w) P splits into the Hermitian parts H1 = (Q + conj Q(-f)) / 2 and H2 = (Q - conj Q(-f)) / 2i,
    Q = H1 + i H2, so IDFT(Q c) = R1 + i R2 with R1, R2 real and w |IDFT(P c)|^2 = R1^2 + R2^2.  The image
    is thus a sum of squares of real fields, sum_j (L h_j)^2, L the real linear map from a Hermitian array to a
    real field, and depends on the 2K arrays h_j (as real vectors [Re | Im]) only through S = sum_j h_j h_j^T.
    With U an orthonormal basis of the range of the Gram matrix h h^T (FP64 eigenvectors whose eigenvalue
    exceeds `tol` of the largest), g = U^T h gives the same S from rank(h) arrays, still Hermitian (real
    combinations).  Two real fields g1, g2 packed as g1 + i g2 give back |IDFT((g1 + i g2) c)|^2 =
    (L g1)^2 + (L g2)^2.  A plane's K fields so become ceil(rank / 2) fields of weight 1.  SOCS kernels of optics
    symmetric under f -> -f span K real dimensions -- degenerate eigenpairs, which an eigensolver returns as
    complex mixtures, included -- so K kernels pack into ceil(K / 2) transforms.  The identity needs nothing of
    the kernels, only a real single-channel mask, and holds for every form of the coherent sum.

    Returns (pupils [Z, K', br, bc] complex64, weights [Z, K'] float32) with planes padded by zero fields of
    weight 0, or None when the band is not centred, a weight is negative, or nothing is gained (K' >= K).
    """
    br, bc = pupils.shape[-2], pupils.shape[-1]
    if not (br % 2 == 1 and bc % 2 == 1 and band.m0r == -(br - 1) // 2 and band.m0c == -(bc - 1) // 2):
        return None
    if bool((weights < 0).any()):
        return None
    q = pupils.to(torch.complex128) * weights.to(torch.float64).sqrt()[..., None, None]
    m = torch.flip(q, dims=(-2, -1)).conj()                            # conj Q(-f) on the centred band
    h = torch.stack(((q + m) / 2, (q - m) / 2j), dim=2).flatten(1, 2)  # [Z, 2K, br, bc], Hermitian
    planes = []
    for z in range(h.shape[0]):
        v = torch.cat((h[z].real, h[z].imag), dim=-1).flatten(1)       # [2K, 2 br bc] real vectors
        sig, u = torch.linalg.eigh((v @ v.T).cpu())                    # the Gram matrix's eigenpairs, on the host
        keep = sig > tol * max(float(sig.max()), 1e-300)
        g = (u[:, keep].T.to(v.device) @ v).view(-1, br, 2 * bc)
        planes.append(torch.complex(g[..., :bc], g[..., bc:]))
    kp = max(1, max((g.shape[0] + 1) // 2 for g in planes))
    if kp >= pupils.shape[1]:
        return None
    out = torch.zeros((len(planes), kp, br, bc), dtype=torch.complex128, device=pupils.device)
    w = torch.zeros((len(planes), kp), dtype=torch.float32, device=pupils.device)
    for z, g in enumerate(planes):
        j = g.shape[0]
        out[z, :(j + 1) // 2] = g[0::2]
        out[z, :j // 2] += 1j * g[1::2]
        w[z, :(j + 1) // 2] = 1.0
    return out.to(torch.complex64).contiguous(), w


class CoherentModel:
    """Fields resident on the device for one optics key and grid: pupils [Z, K, br, bc] complex64 with weights
    [Z, K] on `band`, for a ny x nx grid.  image() of a batch of masks is
        out[b, z] = sum_k w[z, k] |IDFT(P[z, k] .* c_b)|^2        (summed over the masks' channels too)
    -- SOCS kernels of Z focus planes (w = 1, CalculateAerialImage_SOCS.py:3-11) or the Abbe pupils of every
    (source point, field component) (w = n v_j / sum v, CalculateAerialImage.py:46-92).
    """

    def __init__(self, pupils: torch.Tensor, weights: torch.Tensor, band: Band, ny: int, nx: int, kind: str = 'socs',
                 form: str | None = None, pack: bool = True):
        if pupils.dim() != 4 or pupils.shape[2:] != (band.br, band.bc):
            raise ValueError('pupils must be [Z, K, br, bc] on the band')
        if weights.shape != pupils.shape[:2]:
            raise ValueError('weights must be [Z, K]')
        if band.br > ny or band.bc > nx:
            raise ValueError(f'band {band.br}x{band.bc} does not fit the {ny}x{nx} grid')
        self.device = require_cuda(pupils.device)
        self.pupils = pupils.to(self.device, torch.complex64).contiguous()
        self.weights = weights.to(self.device, torch.float32).contiguous()
        if form not in (None,) + FORMS:
            raise ValueError(f'form must be one of {FORMS}')
        if form == 'bf16x3' and not tc_supported(band):
            raise ValueError(f'the bf16x3 form covers bands up to 64 x 64 (this one is {band.br} x {band.bc})')
        self.band, self.ny, self.nx, self.kind, self.form = band, ny, nx, kind, form
        self.plan = Plan.get(ny, nx, band, self.device)
        # the same images from fewer transforms for real single-channel masks (pack_real_fields), or None; it is
        # dropped when the weights change (an Abbe model re-weighted for a new source runs its own fields).  A model
        # built for one call (pack=False) skips it.
        self.packed = pack_real_fields(self.pupils, self.weights, band) if pack else None

    @property
    def planes(self):
        return self.pupils.shape[0]

    @property
    def count(self):
        return self.pupils.shape[1]

    def fields_for(self, kind: int, nch: int = 1):
        """(pupils, weights) the coherent sum of image() uses for masks of this kind: the packed fields for real
        single-channel masks when packing gains, else the model's own."""
        if self.packed is not None and kind in (N.FIELD_REAL_F32, N.FIELD_U8) and nch == 1:
            return self.packed
        return self.pupils, self.weights

    @property
    def nbytes(self):
        return self.pupils.numel() * 8 + self.weights.numel() * 4

    def workspace_bytes(self, batch: int, nch: int = 1, form: str | None = None) -> int:
        """Device bytes one image() call of `batch` masks allocates besides its input and output."""
        b, p = self.band, self.plan
        nz = self.planes
        form = self.form if form is None else form
        split = (field_split(self.count * nch, batch * nz) if p.use_coarse_fft(None)
                 else field_split_sm(self.count * nch, batch * nz) if p.use_coarse256(form)
                 else field_split(self.count * nch, batch * nz * ((p.mr + 15) // 16)))
        if form == 'bf16x3':
            split = tc_parts_bound(batch * nz, self.count * nch)
            p = Plan.get(self.ny, self.nx, b, self.device, coarse=TC_COARSE)
        tiles = batch * nz * p.ny * 512 if form == 'bf16x3' else 0
        return 8 * (batch * nch * p.ny * b.bc + batch * nch * b.br * b.bc + batch * nz * (2 * b.br - 1) * b.bc
                    + batch * nz * b.bc * p.ny) + 4 * split * batch * nz * p.mr * p.mc + tiles

    def _kind(self, masks):
        return {torch.float32: N.FIELD_REAL_F32, torch.uint8: N.FIELD_U8,
                torch.complex64: N.FIELD_COMPLEX_C64}[masks.dtype]

    def image(self, masks: torch.Tensor, kind: int | None = None, nch: int = 1, scale: float = 1.0,
              out: torch.Tensor | None = None, marks=None, form: str | None = None) -> torch.Tensor:
        """Aerial images of a batch of masks -> [B, Z, ny, nx] float32.

        masks: float32 [B, ny, nx] (real transmission), uint8 [B, ny, nx] or complex64 [B, ny, nx, nch].
        `marks`, if a list, receives (stage name, CUDA event) pairs recorded after each native stage.
        `form`: 'fft' (default where supported) or 'dft' picks the transform form of every stage; 'bf16x3' runs
        the coherent contraction in split BF16x3 on the tensor cores (bands up to 64 x 64) and the N-point
        stages in FFT form where supported.  None takes the model's own form (set at construction).
        """
        if kind is None:
            kind = self._kind(masks)
        if form is None:
            form = self.form
        if masks.shape[1] != self.ny or masks.shape[2] != self.nx:
            raise ValueError(f'mask grid {tuple(masks.shape[1:3])} != model grid {(self.ny, self.nx)}')
        _mark(marks, 'start')
        band = band_spectrum(masks.contiguous(), kind, self.plan, nch=nch, scale=scale, form=form)
        _mark(marks, 'band_spectrum')
        pupils, weights = self.fields_for(kind, nch)
        return coherent_image(band, pupils, weights, self.plan, out=out, marks=marks, form=form)


    def image_host(self, masks: torch.Tensor, out: torch.Tensor, chunk: int = 16, check: bool = False,
                   **kw) -> torch.Tensor:
        """image() of a batch held in pinned host memory, written into the pinned host tensor `out` (shaped as
        image() returns it).  The batch is cut into chunks of `chunk` masks; each chunk's copy to the device,
        its images and the copy of its result back run on three streams (copy-in, the current stream, copy-out)
        with events between them, over three rotating device buffer sets kept by the model, so the copies of
        neighbouring chunks -- also across consecutive calls -- overlap each other and the compute; the host
        link then bounds the path.  The current stream waits for the last copy-out before the call returns, so
        synchronising it (or an event recorded on it) covers the results.  With check=True the call waits for
        the batch and raises DeviceWaitError if a kernel's bounded wait expired (the results are then invalid);
        without it, call N.check_device_status after synchronising.  Keyword arguments go to image()."""
        if masks.is_cuda or out.is_cuda:
            raise ValueError('image_host takes host tensors (image() takes device tensors)')
        if not masks.is_pinned() or not out.is_pinned():
            raise ValueError('image_host needs pinned host memory for masks and out')
        if out.shape[0] != masks.shape[0] or out.dtype != torch.float32 or not out.is_contiguous():
            raise ValueError('out must be a contiguous float32 host tensor with one image (set) per mask')
        if chunk <= 0:
            raise ValueError('chunk must be positive')
        dev = self.device
        key = (chunk, masks.dtype, tuple(masks.shape[1:]), tuple(out.shape[1:]))
        pipe = getattr(self, '_host_pipe', None)
        if pipe is None or pipe['key'] != key:
            pipe = {'key': key, 'h2d': torch.cuda.Stream(dev), 'd2h': torch.cuda.Stream(dev), 'next': 0,
                    'slots': [{'d_in': torch.empty((chunk,) + tuple(masks.shape[1:]), dtype=masks.dtype, device=dev),
                               'd_out': torch.empty((chunk,) + tuple(out.shape[1:]), dtype=torch.float32, device=dev),
                               'in_done': torch.cuda.Event(), 'comp_done': torch.cuda.Event(),
                               'out_done': torch.cuda.Event()} for _ in range(3)]}
            self._host_pipe = pipe
        cur = torch.cuda.current_stream(dev)
        masks = masks.contiguous()
        for s0 in range(0, masks.shape[0], chunk):
            c = min(chunk, masks.shape[0] - s0)
            slot = pipe['slots'][pipe['next']]
            pipe['next'] = (pipe['next'] + 1) % 3
            with torch.cuda.stream(pipe['h2d']):
                pipe['h2d'].wait_event(slot['comp_done'])     # the slot's previous chunk has been read
                slot['d_in'][:c].copy_(masks[s0:s0 + c], non_blocking=True)
                slot['in_done'].record(pipe['h2d'])
            cur.wait_event(slot['in_done'])
            cur.wait_event(slot['out_done'])                  # the slot's previous result has been copied out
            self.image(slot['d_in'][:c], out=slot['d_out'][:c], **kw)
            slot['comp_done'].record(cur)
            with torch.cuda.stream(pipe['d2h']):
                pipe['d2h'].wait_event(slot['comp_done'])
                out[s0:s0 + c].copy_(slot['d_out'][:c], non_blocking=True)
                slot['out_done'].record(pipe['d2h'])
        done = torch.cuda.Event()
        done.record(pipe['d2h'])
        cur.wait_event(done)
        if check:
            done.synchronize()
            N.check_device_status('image_host')
        return out


class SocsKernels(CoherentModel):
    """SOCS kernels of one focus plane resident on the device in band form: [K, br, bc] complex64.

    This is the engine's form of the reference's full-grid kernel array (DecomposeTCC_SOCS.py:26-35): the same
    values, with only the band that can be non-zero kept.  image() returns [B, ny, nx].
    """

    def __init__(self, kernels: torch.Tensor, band: Band, ny: int, nx: int):
        if kernels.dim() != 3 or kernels.shape[1:] != (band.br, band.bc):
            raise ValueError('kernels must be [K, br, bc] on the band')
        k = kernels.shape[0]
        super().__init__(kernels.unsqueeze(0), torch.ones((1, k), device=kernels.device), band, ny, nx, 'socs')
        self.kernels = self.pupils[0]

    @classmethod
    def from_full_grid(cls, kernels: torch.Tensor) -> 'SocsKernels':
        """Band form of a reference-layout kernel array [Ny, Nx, K] (frequency m at index m mod N)."""
        ny, nx = kernels.shape[0], kernels.shape[1]
        dev = require_cuda(kernels.device if kernels.is_cuda else None)
        k = kernels.to(dev)
        nzr = (k != 0).any(dim=2)
        r0, br = cyclic_support(nzr.any(dim=1))
        c0, bc = cyclic_support(nzr.any(dim=0))
        band = Band(centred(r0, ny), br, centred(c0, nx), bc)
        kb = torch.roll(k, shifts=(-band.m0r, -band.m0c), dims=(0, 1))[:br, :bc, :].permute(2, 0, 1)
        return cls(kb.to(torch.complex64).contiguous(), band, ny, nx)

    def image(self, masks: torch.Tensor, kind: int | None = None, nch: int = 1, scale: float = 1.0,
              out: torch.Tensor | None = None, marks=None, form: str | None = None) -> torch.Tensor:
        """SOCS aerial images of a batch of masks -> [B, ny, nx] float32 (see CoherentModel.image)."""
        o = None if out is None else out.view(masks.shape[0], 1, self.ny, self.nx)
        img = super().image(masks, kind=kind, nch=nch, scale=scale, out=o, marks=marks, form=form)
        return img.view(masks.shape[0], self.ny, self.nx)
