// Test harness (host code): the retry chain's inversions of
// harm_ramt_b200/csrc/harm_tryagain.cuh compiled for the CPU, called one
// zone at a time by tests/test_tryagain.py and compared with the
// reference's own methods (Utoprimgen_pick) bit for bit.
#include <math.h>
#include <string.h>

#include "../harm_ramt_b200/csrc/harm_tryagain.cuh"

using namespace harm;

namespace {

Geo<double> geo_of(const double* gcov16, const double* gcon16, double gdet)
{
  Geo<double> g;
  for (int a = 0; a < 4; a++)
    for (int b = a; b < 4; b++) {
      g.gcov[sym(a, b)] = gcov16[a * 4 + b];
      g.gcon[sym(a, b)] = gcon16[a * 4 + b];
    }
  g.g = gdet;
  return g;
}

}  // namespace

extern "C" {

// one method of the chain (ta::M_*) on U in the evolved form (with
// sqrt(-g)); pr: guess in, result out.  Returns the pflag code, -1000 for a
// method not built.
int ta_pick(int which, const double* gcov16, const double* gcon16, double gdet, double gam, double gammafail,
            const double* Uev, double* pr)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  double Ug[NPR];
  ta::evolved_to_geomfree(Uev, g, Ug);
  if (which == ta::M_2D || which == ta::M_LDZ) return -1000;
  return ta::pick(which, Ug, g, gam, gammafail, pr);
}

// the retry chain after a primary 2D result (pr, pfl) from the guess pr0
int ta_chain(const double* gcov16, const double* gcon16, double gdet, double gam, double gammafail, const double* Uev,
             const double* pr0, double* pr, int pfl)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  return ta::tryagain_chain(Uev, g, gam, gammafail, pr0, pr, pfl);
}

// U in the evolved form (primtoU(UEVOLVE)) of the primitives p
void ta_primtoU(const double* gcov16, const double* gcon16, double gdet, double gam, const double* p, double* Uev)
{
  const Geo<double> g = geo_of(gcov16, gcon16, gdet);
  State<double> q;
  state_of(p, g, q);
  flux_of<double, false>(p, q, 0, g, gam, Uev);
}

}  // extern "C"
