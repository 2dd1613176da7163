// cli_defaults.h -- settings the command-line programs share.
#pragma once

// The block solver's filter degree cap when parameters.txt gives none
// (filter_deg): the best degree measured for the production lattice sizes
// (24^3 and 32^3: 60; 48^3: 48); small lattices keep the library default,
// which they converge with in a few passes.  `autotune = N` in laph_ev_ts
// measures it for the run's own batch instead.
inline int default_filter_deg(int L, int library_default) { return L >= 40 ? 48 : (L >= 20 ? 60 : library_default); }
