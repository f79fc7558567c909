// The GPU context of the drop-in shims, built from the reference driver's
// structures (see shim_desc.cpp).  Compiled as C++ against the reference's
// headers.
#pragma once

#include "capacmd.h"
#include "typedef.h"

// The process's context, created on the first call from the structures
// given.  mi, rs and m may be NULL (a shim whose reference signature lacks
// them): molecule ranges then follow from atom_info, and a context made
// without run settings or metal serves RATTLE only; it is made again the
// first time a call brings both.
capac_ctx *shim_context(const Topol *t, const Atom_Info *ai, const Mol_Info *mi, const RunSet *rs, const Metal *m,
                        const System *s);
// The context if one exists, else NULL; and the description it was made from.
capac_ctx *shim_existing();
const capac_desc *shim_desc();
// Print the library's message for a failed call and exit(1), as the
// reference does on its own errors.
void shim_fail(const char *what);
