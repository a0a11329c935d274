"""Splitting a difference between two GPU evaluations of ComputeBilateralNCC
(HPM.cu:325-397) into its two causes.

Both evaluations report the 36 source samples of each window (the product's
hpm_tap_samples, the reference shim's hpm_ref_tap_samples).  Where the
texture unit rounded a tap coordinate of one of them to another 1/256 step,
the samples differ; the exact effect of that is the float64 NCC of one
side's samples minus the float64 NCC of the other's.  What remains,

    residual = (cost_a - cost_b) - (ncc64(samples_a) - ncc64(samples_b)),

is the FP32 evaluation of the same samples, which the tests hold to 1e-4
relative with no exceptions.
"""
import numpy as np

OFFS = np.array([(i, j) for i in range(-5, 6, 2) for j in range(-5, 6, 2)])  # tap order (i outer, j inner)


def ref_window(ref_img, pixels):
    """Reference-window pixels (n, 36) and bilateral weights (n, 36) in
    float64, with the reference's clamped integer texel reads."""
    h, w = ref_img.shape
    px, py = pixels % w, pixels // w
    xs = np.clip(px[:, None] + OFFS[None, :, 0], 0, w - 1)
    ys = np.clip(py[:, None] + OFFS[None, :, 1], 0, h - 1)
    r = ref_img[ys, xs].astype(np.float64)
    rc = ref_img[py, px].astype(np.float64)[:, None]
    sd = np.sqrt((OFFS ** 2).sum(-1)).astype(np.float64)[None, :]
    wgt = np.exp(-sd / (2 * 5.0 ** 2) - np.abs(r - rc) / (2 * 3.0 ** 2))
    return r, wgt


def ncc64(r, wgt, s):
    """NCC cost in float64 of samples s (n, S, 36) against windows (n, 36)."""
    W = wgt.sum(-1)[:, None]
    wn = (wgt / W)[:, None, :]
    rr = r[:, None, :]
    mr, mrr = (wn * rr).sum(-1), (wn * rr * rr).sum(-1)
    ms, mss, mrs = (wn * s).sum(-1), (wn * s * s).sum(-1), (wn * rr * s).sum(-1)
    var_r, var_s = mrr - mr * mr, mss - ms * ms
    cov = mrs - mr * ms
    with np.errstate(invalid="ignore", divide="ignore"):
        c = 1.0 - cov / np.sqrt(var_r * var_s)
    c = np.clip(c, 0.0, 2.0)
    return np.where((var_r < 1e-5) | (var_s < 1e-5), 2.0, c)


def split(cost_a, cost_b, samples_a, samples_b, inside_a, inside_b, ref_img, pixels):
    """(crossed, effect, residual) per (pixel, view): crossed where any tap
    sample differs; effect = exact change those samples cause; residual =
    the rest of cost_a - cost_b.  Where one side has the centre outside and
    the other inside, crossed is True and effect takes the whole difference."""
    r, wgt = ref_window(ref_img, pixels)
    sa, sb = samples_a.astype(np.float64), samples_b.astype(np.float64)
    d = cost_a.astype(np.float64) - cost_b.astype(np.float64)
    both_in = inside_a & inside_b
    crossed = (samples_a != samples_b).any(-1) & both_in
    effect = np.where(crossed, ncc64(r, wgt, sa) - ncc64(r, wgt, sb), 0.0)
    flip = inside_a != inside_b
    effect = np.where(flip, d, effect)
    crossed = crossed | flip
    return crossed, effect, d - effect


MARGIN = 1.25  # first-order bounds: 25 % for the second-order terms they leave out


def exact_costs(samples, inside, ref_img, pixels):
    """float64 NCC (n, S) of the given tap samples (n, S, 36), 2 where the
    window centre falls outside the source view: the exact value both FP32
    evaluations of the same samples approximate."""
    r, wgt = ref_window(ref_img, pixels)
    return np.where(inside, ncc64(r, wgt, samples.astype(np.float64)), 2.0)


def _offenders(over, got, ref, bound, exact, extra):
    idx = np.argsort(-np.where(over, np.abs(got - ref) - bound, -np.inf).ravel())[:min(5, int(over.sum()))]
    rows = []
    for i in idx:
        row = f"#{i}: got {got.flat[i]:.7f} ref {ref.flat[i]:.7f} bound {bound.flat[i]:.3g}"
        if exact is not None:
            row += f" exact {exact.flat[i]:.7f} (got-exact {got.flat[i] - exact.flat[i]:.3g}, " \
                   f"ref-exact {ref.flat[i] - exact.flat[i]:.3g})"
        for k, v in (extra or {}).items():
            row += f" {k} {np.asarray(v).flat[i]:.4g}"
        rows.append(row)
    return "; ".join(rows)


def fp32_bound(r, wgt, s):
    """First-order bound of ONE FP32 evaluation's error against the float64
    NCC of the same samples s (n, S, 36), the oracle's model of it
    (or_ncc_bounds_px, oracle/hpm_oracle.c) evaluated on these very samples:
    window sums within 16 units of 2^-24 (rows of 6 taps, all terms
    positive), the variances and covariance cancelling, and a relative
    error of 1e-5 on every bilateral weight.  Returns (bound, flip): flip
    marks windows whose variance lies within its own error bound of the
    1e-5 cut, where an FP32 evaluation may take the other branch."""
    u = 2.0 ** -24
    g = 16.0 * u
    W = wgt.sum(-1)[:, None, None]
    w = wgt[:, None, :]
    rr = r[:, None, :]
    mr, mrr = (w * rr).sum(-1) / W[..., 0], (w * rr * rr).sum(-1) / W[..., 0]
    ms, mss, mrs = (w * s).sum(-1) / W[..., 0], (w * s * s).sum(-1) / W[..., 0], (w * rr * s).sum(-1) / W[..., 0]
    var_r, var_s = mrr - mr * mr, mss - ms * ms
    cov = mrs - mr * ms
    e_vr = g * mrr + 2 * mr * g * mr + u * (mrr + mr * mr)
    e_vs = g * mss + 2 * ms * g * ms + u * (mss + ms * ms)
    e_cov = g * mrs + mr * g * ms + ms * g * mr + u * (mrs + mr * ms)
    with np.errstate(invalid="ignore", divide="ignore"):
        vv = np.sqrt(var_r * var_s)
        e_c = e_cov / vv + np.abs(cov) / vv * (0.5 * (e_vr / var_r + e_vs / var_s) + u) + u
        dmr, dms = (rr - mr[..., None]) / W, (s - ms[..., None]) / W
        dmrr, dmss = (rr * rr - mrr[..., None]) / W, (s * s - mss[..., None]) / W
        dmrs = (rr * s - mrs[..., None]) / W
        dvr = dmrr - 2 * mr[..., None] * dmr
        dvs = dmss - 2 * ms[..., None] * dms
        dcov = dmrs - mr[..., None] * dms - ms[..., None] * dmr
        dc = -(dcov / vv[..., None] - cov[..., None] / (2 * vv[..., None]) *
               (dvr / var_r[..., None] + dvs / var_s[..., None]))
        e_w = (np.abs(dc) * 1e-5 * w).sum(-1)
    flip = (np.abs(var_r - 1e-5) <= 2 * e_vr) | (np.abs(var_s - 1e-5) <= 2 * e_vs)
    bound = np.where((var_r < 1e-5) | (var_s < 1e-5), 0.0, e_c + e_w)
    return bound, flip


def check_exact(got, samples, inside, ref_img, pixels, what):
    """An FP32 evaluation against the float64 NCC of its own samples: within
    1e-4 max(1, |exact|) + MARGIN * fp32_bound everywhere, except windows
    where the flat-window branch may flip (fp32_bound's flip)."""
    r, wgt = ref_window(ref_img, pixels)
    s = samples.astype(np.float64)
    exact = np.where(inside, ncc64(r, wgt, s), 2.0)
    bound, flip = fp32_bound(r, wgt, s)
    got = np.asarray(got, np.float64).reshape(exact.shape)
    d = np.abs(got - exact)
    over = (d > 1e-4 * np.maximum(1.0, np.abs(exact)) + MARGIN * np.nan_to_num(bound, nan=np.inf)) & ~flip & inside
    assert not over.any(), (f"{what}: {int(over.sum())} values off the exact NCC of their samples, worst "
                            f"{float(d[over].max()):.3g} (bound {float(bound[over][np.argmax(d[over])]):.3g})")


SELF_INCONSISTENT_CAP = 1e-3  # at most this fraction of a field's values may be exempted


def reference_self_inconsistent(ref, exact, bound):
    """Values where the reference's NCC kernel lies beyond the tap-crossing
    bound of the exact NCC of the samples that the reference's own
    coordinate functions give (hpm_ref_tap_samples): the reference disagrees
    with itself there, by more than any crossing of a weight step explains
    (measured: 2 of 16,384 values of the 640x480 case, 4.4e-3 and 1.4e-3 off
    its own samples; the oracle, whose coordinates round on their own, lands
    where the reference's kernel does).  Returns the mask; at most
    SELF_INCONSISTENT_CAP of the values may be in it."""
    ref, exact = np.asarray(ref, np.float64), np.asarray(exact, np.float64)
    bound = np.broadcast_to(np.asarray(bound, np.float64), ref.shape)
    off = np.abs(ref - exact) > 1e-4 * np.maximum(1.0, np.abs(ref)) + MARGIN * bound
    assert off.mean() <= SELF_INCONSISTENT_CAP, (
        f"the reference's kernel is off its own samples in {int(off.sum())} of {off.size} values")
    return off


def check_within_bound(got, ref, bound, what, exact=None, extra=None, exempt=None):
    """|got - ref| <= 1e-4 max(1, |ref|) + MARGIN * bound for every value
    outside `exempt` (a mask from reference_self_inconsistent, whose values
    the caller checks against the exact NCC instead), and <= 1e-4 max(1,
    |ref|) alone where the bound is below 1e-4 (well conditioned).  Returns
    the fraction of values within 1e-4.  exact (the float64 value of the
    same samples) and extra arrays only enrich the message of a failure."""
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    bound = np.broadcast_to(np.asarray(bound, np.float64), got.shape)
    d = np.abs(got - ref)
    tol = 1e-4 * np.maximum(1.0, np.abs(ref))
    over = d > tol + MARGIN * bound
    if exempt is not None:
        over &= ~np.asarray(exempt, bool).reshape(over.shape)
    assert not over.any(), (f"{what}: {int(over.sum())} values beyond the bound, worst excess "
                            f"{float((d - tol - MARGIN * bound).max()):.3g}; "
                            + _offenders(over, got, ref, MARGIN * bound + tol, exact, extra))
    calm = bound < 1e-4
    if exempt is not None:
        calm &= ~np.asarray(exempt, bool).reshape(calm.shape)
    assert (d[calm] <= tol[calm]).all(), f"{what}: {int((d[calm] > tol[calm]).sum())} well-conditioned values off"
    return float((d <= tol).mean())
