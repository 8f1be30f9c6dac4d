"""Fortran edit descriptors as gfortran writes them, for comparing the text
files the driver writes (CHKP, CHKJ) with what the reference's WRITE
statements produce (AWP-ODC-SGT/src/io.f:481-536, pmcl3d.f:1478-1479).
Written from the Fortran standard's rules for E, F, G and I editing; it
shares no code with the driver's C formatter."""


def _digits(x, d):
    """Decimal digits and exponent of |x| rounded to d significant digits:
    |x| ~ 0.DIGITS * 10**exp."""
    s = "%.*e" % (d - 1, abs(float(x)))
    mant, ex = s.split("e")
    return mant.replace(".", ""), int(ex) + 1


def e(x, w, d):
    """Ew.d: [-]0.ddddE+xx, right-justified in w columns."""
    x = float(x)
    if x == 0.0:
        body = "0." + "0" * d + "E+00"
    else:
        dig, ex = _digits(x, d)
        body = "%s0.%sE%s%02d" % ("-" if x < 0 else "", dig, "-" if ex < 0 else "+", abs(ex))
    if len(body) > w and body.lstrip("-").startswith("0."):
        body = body.replace("0.", ".", 1)       # the optional leading zero goes first
    return "*" * w if len(body) > w else body.rjust(w)


def f(x, w, d):
    """Fw.d."""
    s = "%.*f" % (d, float(x))
    return "*" * w if len(s) > w else s.rjust(w)


def g(x, w, d):
    """Gw.d: F editing with d - k decimals and four blanks when the value
    rounded to d significant digits lies in [0.1, 10**d) (k = its number of
    integer digits), else Ew.d."""
    x = float(x)
    if x == 0.0:
        return f(0.0, w - 4, d - 1) + "    "
    _, k = _digits(x, d)
    if 0 <= k <= d:
        return f(x, w - 4, d - k) + "    "
    return e(x, w, d)


def i(n, w):
    """Iw."""
    s = "%d" % n
    return "*" * w if len(s) > w else s.rjust(w)


def list_directed(*items):
    """gfortran list-directed output of character and default-integer items:
    a leading blank, integers as I11 after a blank separator, strings as
    they are."""
    out = " "
    for k, it in enumerate(items):
        if isinstance(it, str):
            out += it
        else:
            out += (" " if k else "") + i(it, 11)
    return out
