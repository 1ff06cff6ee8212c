// ERF_PlaneAverage.H stand-in -- TEST INFRASTRUCTURE ONLY.  The Kessler
// initialisation file includes the plane-average utility without using it;
// the operators pinned here need none of it.
#pragma once
