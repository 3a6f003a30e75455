// B200 drop-in for the reference solver's outer iteration.
//
// A maintainer adds b200_dropin.cpp to the reference build (next to
// Utilities/iterations.cpp), links libcps.so, and branches at the top of
// SIMPLE::calculateStep (Utilities/iterations.cpp:82):
//
//     if (pressureSolverType >= 5) return b200StepDropIn(*this, pressureIterations);
//
// pressureSolverType is the reference's solver registry member (SIMPLE.h:145,
// 0..4 today); 5 selects this path in FP64, 6 in mixed precision (FP32 inner
// Jacobi and PCG inside an FP64 defect correction; same fixed point).  The
// design's fields live on the GPU between steps; b200SyncFieldsToHost copies
// them back into the SIMPLE object for saveAll / checkpoints
// (SIMPLE.cpp:432-443), and b200SamplePlaneAtX replaces samplePlaneAtX
// (postprocessing.cpp:97-230) in the per-iteration pressure-drop monitor so no
// field leaves the GPU per step.
//
// Design identity.  Every SIMPLE object has its own device design, so several
// objects (several designs of one grid, say) can be stepped in one process.
// A step rebuilds the object's device design from the host object, uploading
// alpha, gamma, u, v and p, when
//   * it is the first step of that object,
//   * a new object was constructed at the address of a released or destroyed
//     one (its residU/residV/residMass are back at their constructor values
//     instead of the ones the last step wrote), or
//   * a solver parameter it was built from changed (grid, spacings, fluid,
//     relaxation, inner tolerances and caps, convection scheme, 2.5-D
//     settings, pseudo-transient settings, precision).
// Editing alpha, gamma, u, v or p of an object in place between steps (a new
// density field in a design loop, a restart load) is announced with
// b200Invalidate(s): the host's arrays are uploaded before the next step.
// runIterations calls it once at its top, so every run starts from the host
// object's state, as the reference's own loop does.
#pragma once

#include "SIMPLE.h"

// One outer iteration on the GPU; returns max(residU, residV, residMass) and
// sets residU/residV/residMass and pressureIterations like calculateStep
// (iterations.cpp:125-127, 451, 525).  Throws std::runtime_error with the
// library's message when the GPU path fails (it never falls back to the CPU).
decltype(SIMPLE::hx) b200StepDropIn(SIMPLE& s, int& pressureIterations);

// The host's alpha, gamma, u, v and p of s are uploaded before its next step
// (call after changing them in place).
void b200Invalidate(const SIMPLE& s);

// Copy u, v, p, pStar, uStar, vStar, dE, dN from the GPU into s.
void b200SyncFieldsToHost(SIMPLE& s);

// samplePlaneAtX computed on the GPU from the resident fields (the host
// object's own state is uploaded first if s has no current device design).
PlaneMetrics b200SamplePlaneAtX(const SIMPLE& s, decltype(SIMPLE::hx) xPhysical);

// Release the device design of s (call before s is destroyed, or at any time:
// the next step rebuilds it from the host object).
void b200Release(const SIMPLE& s);

// Release every device design (call once at exit).
void b200Release();
