// transport_gpu.h -- the reference's `transport` class
// (src/transport/transport.h:45-320) running its step on the B200 library
// through the C ABI of include/sedona_gpu.h.
//
// This is the code a maintainer adds to the reference: `attach` belongs at
// the end of transport::init (src/transport/transport_init.cpp:427) and
// `step` replaces the body of transport::step (src/transport/transport.cpp:
// 26-140) up to the temperature solve.  Here they are free functions over a
// `transport&`, compiled against the reference's own headers; the reference
// declares the members they read private, so the translation unit is
// compiled with them opened (the member-function form needs nothing of the
// kind).
//
// The transport keeps owning its vectors: `step` flattens the zone state into
// the ABI's structure-of-arrays structs and copies the results back into the
// same vectors the reference writes out (J_nu_, the zones' e_abs, e_rad,
// f*_rad, the opacity tables, planck/rosseland means, eps_imc, n_elec,
// optical_spectrum flux/click), so write_radiation_file and
// spectrum_array::print work unchanged.
#pragma once
#include "sedona_gpu.h"

class transport;
class ParameterReader;

namespace sed_binding {

struct GpuTransport;

// Creates the context for `t` (after transport::init): parameters, grids,
// opacity switches and the atomic data the transport loaded.  precision is
// enum sed_precision; device -1 uses the current device.  Null on failure,
// with the message in last_error(nullptr).
GpuTransport* attach(transport& t, ParameterReader* params, int precision, int device);

// One transport step of dt on the device: zone state up, sed_step (opacity
// build, emission, propagation, normalisation), results back into t.
// Returns the sed_status of the step; stats may be null.
int step(transport& t, GpuTransport* g, double dt, sed_step_stats* stats);

const char* last_error(GpuTransport* g);
void detach(GpuTransport* g);

}  // namespace sed_binding
