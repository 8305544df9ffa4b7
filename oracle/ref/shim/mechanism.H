// Species count for the oracle/_ref build; set per build with -DPCG_REF_NS=<n>.
#pragma once
#ifndef PCG_REF_NS
#error "PCG_REF_NS must be defined"
#endif
#define NUM_SPECIES PCG_REF_NS
