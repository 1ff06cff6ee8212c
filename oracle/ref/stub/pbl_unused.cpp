// pbl_unused.cpp -- TEST INFRASTRUCTURE ONLY.  ComputeTurbulentViscosity
// dispatches to the PBL schemes (declared in PBL/ERF_PBLModels.H) when
// pbl_type is not None; the operators pinned here run with pbl_type None,
// so the two schemes are defined to abort instead of being compiled from
// their sources (which need the whole MOST surface-layer object).
#include <AMReX_MultiFab.H>
#include "ERF_IndexDefines.H"
#include "ERF_EddyViscosity.H"
#include "ERF_Diffusion.H"
#include "ERF_PBLModels.H"

void ComputeDiffusivityMYNN25(const amrex::MultiFab&, const amrex::MultiFab&, const amrex::MultiFab&,
                              amrex::MultiFab&, const amrex::Geometry&, const TurbChoice&,
                              std::unique_ptr<ABLMost>&, bool, int, const amrex::BCRec*, bool,
                              const std::unique_ptr<amrex::MultiFab>&, const int, const int) {
    amrex::Abort("MYNN2.5 PBL is not part of the pinned operators");
}

void ComputeDiffusivityYSU(const amrex::MultiFab&, const amrex::MultiFab&, const amrex::MultiFab&, amrex::MultiFab&,
                           const amrex::Geometry&, const TurbChoice&, std::unique_ptr<ABLMost>&, bool, int,
                           const amrex::BCRec*, bool, const std::unique_ptr<amrex::MultiFab>&) {
    amrex::Abort("YSU PBL is not part of the pinned operators");
}
