/*
 * exp_shim.cpp -- TEST INFRASTRUCTURE: exp(x) correctly rounded for the
 * ConcZ oracle.
 *
 * Linked into oracle/_ref/yz_probe_cz ahead of the C library, this definition
 * of exp takes the place of the libm's for every call the reference's sources
 * make (the property laws base * exp(k (c - c0)), FluidProperty.h:176-180):
 * the reference's numerics then no longer depend on which arguments the host's
 * libm misrounds (about one in 1,300), and the device's ConcZ step, which uses
 * the same correctly rounded function (yuzen_b200/csrc/yz_exp.h), can be held
 * to them bit for bit.  oracle/_ref/yz_probe_cz_libm is the same probe with the
 * libm's exp (the reference exactly as it builds: its CPU timing, and the
 * check that the device stays within the solve's conditioning of it).
 */
#include "yz_exp.h"

extern "C" double exp(double x) { return yz::crexp::Exp(x); }
