// ERF_TurbPertStruct.H stand-in -- TEST INFRASTRUCTURE ONLY.  SolverChoice
// includes the turbulent-inflow perturbation header but holds no member of
// its types; the operators pinned here do not use it.
#pragma once
