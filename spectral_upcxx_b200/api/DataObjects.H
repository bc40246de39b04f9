#ifndef _DATA_OBJECTS_H_
#define _DATA_OBJECTS_H_

// Umbrella header of the field API (the reference's src/DataObjects.H).

#include <array>
#include <complex>
#include <upcxx/upcxx.hpp>
#include <vector>

class Vector;

#include "Scalar.H"
#include "Vector.H"
#include "Operators.H"

// Runtime settings of the B200 field API (no reference counterpart).
namespace sns_api {
/// storage precision of new fields: SNS_C128 (default) or SNS_C64
/// (environment SNS_PRECISION=fp32 selects SNS_C64 at start-up)
int precision();
void set_precision(int prec);
/// Nyquist zeroing after every forward transform (the reference's ZERO
/// build flag, on by default; environment SNS_ZERO=0 turns it off)
bool zero_high_modes();
void set_zero_high_modes(bool on);
/// wait for queued device work
void synchronize();
}  // namespace sns_api

#endif
