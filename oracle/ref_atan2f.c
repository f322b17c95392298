/*
 * ref_atan2f.c - patch P4 of the reference build (TEST INFRASTRUCTURE ONLY).
 *
 * Linked into oracle/_ref/ref_cr and ref_unstable: the reference's std::atan2(float, float)
 * calls (MathUtils.h:39, Tracklet.cxx:36) resolve to this definition instead of the C library's,
 * so the reference computes the correctly rounded azimuths the device computes.
 */
#include "../include/itsu_atan2f.h"

float atan2f(float y, float x);
float itsu_ref_cr_atan2f(float y, float x);

float atan2f(float y, float x) { return itsu_atan2f(y, x); }

/* Same function under its own name: the harness checks that atan2f resolves to it. */
float itsu_ref_cr_atan2f(float y, float x) { return itsu_atan2f(y, x); }
