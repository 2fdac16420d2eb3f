"""oercel_b200: the 2D DPD step with lipid chemistry of the Oercel engine on B200.

The step runs in libdpd.so (hand-written sm_100a CUDA, C ABI in include/dpd.h);
this package is the host side: parameters with the reference's keys, the
in-process Engine, and the drop-in command-line front end.
"""
from ._capi import DpdError, load
from .engine import EVENT_KINDS, Engine, make_soup, soup_for
from .params import ParamError, Params

__all__ = ["DpdError", "Engine", "EVENT_KINDS", "ParamError", "Params", "load", "make_soup", "soup_for"]
