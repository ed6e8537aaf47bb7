/*
 * ref_ewald.cpp -- TEST INFRASTRUCTURE (oracle).  Compiles the reference's
 * examples/Ewald.C (EwaldData::EwaldInit, the reciprocal-space table built
 * from the root cell's moments) where it lies, without Charm++: the build
 * defines EXAMPLE_MAIN_H so that examples/Main.h contributes nothing, and
 * ref_shim/paratreet.decl.h stands in for the generated CBase_EwaldData.
 * fPeriod and nReplicas are defined in ref_driver.cpp.
 */
#include "common.h"
#include "Particle.h"
#include "CentroidData.h"
#include "EwaldData.h"
#include "Ewald.C"
