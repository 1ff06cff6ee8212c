// AMReX_PhysBCFunct.H -- TEST INFRASTRUCTURE ONLY: forwards to the single-box AMReX stand-in.
#pragma once
#include "amrex_shim_core.H"
