// B200 drop-in for the reference solver's outer iteration.
//
// A maintainer adds b200_dropin.cpp to the reference build (next to
// Utilities/iterations.cpp), links libcps.so, and branches at the top of
// SIMPLE::calculateStep (Utilities/iterations.cpp:82):
//
//     if (pressureSolverType == 5) return b200StepDropIn(*this, pressureIterations);
//
// pressureSolverType is the reference's solver registry member (SIMPLE.h:145,
// 0..4 today); 5 selects this path.  The design's fields live on the GPU
// between steps; b200SyncFieldsToHost copies them back into the SIMPLE
// object for saveAll / checkpoints (SIMPLE.cpp:432-443), and
// b200SamplePlaneAtX replaces samplePlaneAtX (postprocessing.cpp:97-230) in the
// per-iteration pressure-drop monitor so no field leaves the GPU per step.
#pragma once

#include "SIMPLE.h"

// One outer iteration on the GPU; returns max(residU, residV, residMass) and
// sets residU/residV/residMass and pressureIterations like calculateStep
// (iterations.cpp:125-127, 451, 525).  Throws std::runtime_error with the
// library's message when the GPU path fails (it never falls back to the CPU).
decltype(SIMPLE::hx) b200StepDropIn(SIMPLE& s, int& pressureIterations);

// Copy u, v, p, pStar, uStar, vStar, dE, dN from the GPU into s.
void b200SyncFieldsToHost(SIMPLE& s);

// samplePlaneAtX computed on the GPU from the resident fields.
PlaneMetrics b200SamplePlaneAtX(const SIMPLE& s, decltype(SIMPLE::hx) xPhysical);

// Release the device state (call once at exit; a new grid size also replaces it).
void b200Release();
