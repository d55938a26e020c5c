"""Energy tolerance of the parity tests.

The bar is 1e-5 relative per term.  Terms that are sums of contributions of
both signs (ele, and vdw/pmf/psp/hdb in general) are compared against the sum
of |contribution| (computed by the oracle), so that cancellation to near zero
does not turn rounding noise into a failure:

    |gpu - ref| <= RTOL * max(|ref|, scale) + ATOL

For the normalised terms a*e + b the scale is |a| * scale_raw + |b| plus one
float ulp of that magnitude; for the weighted total it is sum |w_i| scale_i.
"""
import numpy as np

RTOL = 1e-5
ATOL = 1e-7


def raw_scale(raw_ref, abs_sum):
    s = np.abs(raw_ref).copy()
    s[:, :5] = np.maximum(s[:, :5], abs_sum[:, :5])
    return s


def check_raw(raw_gpu, raw_ref, abs_sum, rtol=RTOL):
    scale = raw_scale(raw_ref, abs_sum)
    err = np.abs(raw_gpu - raw_ref)
    bad = err > rtol * scale + ATOL
    return bad, err / (scale + 1e-300)


def check_terms(terms_gpu, terms_ref, raw_ref, abs_sum, ff, rtol=RTOL):
    a = np.asarray(ff.a_para, np.float64)[:9]
    b = np.asarray(ff.b_para, np.float64)[:9]
    w = np.asarray(ff.w, np.float64)[:9]
    scale_raw = raw_scale(raw_ref, abs_sum)
    scale = np.zeros_like(terms_ref, dtype=np.float64)
    scale[:, :9] = np.abs(a) * scale_raw + np.abs(b)
    scale[:, 9] = (np.abs(w) * scale[:, :9]).sum(axis=1)
    ulp = np.spacing(np.abs(terms_ref).astype(np.float32)).astype(np.float64) * 4
    err = np.abs(terms_gpu.astype(np.float64) - terms_ref.astype(np.float64))
    bad = err > rtol * np.maximum(np.abs(terms_ref), scale) + ulp
    return bad, err / (scale + 1e-300)
