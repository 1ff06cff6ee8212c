// ERF_ABLMost.H stand-in -- TEST INFRASTRUCTURE ONLY.  The operators pinned
// here take the MOST surface-layer object only as an unused argument (the
// configurations have no MOST boundary), so an empty class replaces
// BoundaryConditions/ERF_ABLMost.H and its dependency tree.
#pragma once
#include <AMReX_MultiFab.H>
class ABLMost {};
