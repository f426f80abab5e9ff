// Test infrastructure for the oracle build only (never shipped, never linked into the product).
//
// The reference painter path names mpz_class / mpf_class only inside type traits
// (src/com/type/trait.h:20-37) and inside templates that the painter never instantiates
// (src/geometry/core/linear_algebra.h:29,290-310). GMP headers are not installed on this
// machine, so these two empty types stand in for them while the reference painter sources
// are compiled in place.
#pragma once

class mpz_class
{
};

class mpf_class
{
};
