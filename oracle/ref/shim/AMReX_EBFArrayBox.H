// Forwarding header of the AMReX-API shim (oracle/_ref build only).
#pragma once
#include "pcg_amrex_shim.H"
