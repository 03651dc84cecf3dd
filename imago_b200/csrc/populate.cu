// populate.cu -- the state populations of one SCF step, on the host
// (populateStates, populate.F90:150-620).
//
// populateStandard (populate.F90:190-483): the numStates x numKPoints x spin
// eigenvalues, listed k-point by k-point, spin by spin, state fastest, are
// sorted ascending (stably); each state in turn takes kPointWeight(k) / spin
// electrons until numElectrons are placed, the last one the remainder; the
// states within smallThresh of that energy then share the charge placed
// among them in proportion to their weights.  The gap to the next state
// classifies the system (metal below metalGapThresh, direct when the two
// states share a k-point, indirect otherwise).
//
// populateSmearing (populate.F90:486-620), for a non-zero thermalSigma:
// the Fermi level is bisected, at most 500 times, between the highest
// occupied energy minus fermiSearchLimit and the next energy plus it; every
// state takes its weight times stepFunction((E - E_F) / thermalSigma,
// maxThermalRange) (mathSubs.f90:164-185), the sum stopping at the first
// state the step function zeroes, until the charge is within smallThresh
// of numElectrons.
//
// Host work over a few hundred thousand values at most: done where the
// eigenvalues are read, with the reference's summation order.
#include <algorithm>
#include <climits>
#include <cmath>
#include <numeric>
#include <vector>

#include "intg.cuh"

namespace {

constexpr double kSmallThresh = 1.0e-8;     // constants.f90:49
constexpr double kMetalGapThresh = 1.0e-3;  // populate.F90, metalGapThresh
constexpr int kFermiSteps = 500;

double step_function(double x, double range) {
  if (x > range) return 0.0;
  if (x < -range) return 1.0;
  return 1.0 / (1.0 + std::exp(x));
}

}  // namespace

extern "C" int imago_populate_states_sorted(
    int num_kpoints, int spin, int num_states, const double *eigenvalues,
    const double *kpoint_weights, double num_electrons, double thermal_sigma,
    double max_thermal_range, double fermi_search_limit, double *population, double *info,
    double *sorted_energies, int *sort_index) {
  if (num_kpoints <= 0 || spin < 1 || spin > 2 || num_states <= 0 || !eigenvalues ||
      !population || !info || !(num_electrons >= 0.0) || !(thermal_sigma >= 0.0))
    return IMAGO_ERR_INVALID;
  const long long n = (long long)num_kpoints * spin * num_states;
  if (sort_index && n > (long long)INT_MAX) return IMAGO_ERR_RANGE;
  const long long per_k = (long long)spin * num_states;
  std::vector<double> kw(num_kpoints);
  for (int k = 0; k < num_kpoints; ++k)
    kw[k] = kpoint_weights ? kpoint_weights[k] : 2.0 / num_kpoints;
  std::vector<long long> order(n);
  std::iota(order.begin(), order.end(), 0LL);
  std::stable_sort(order.begin(), order.end(), [&](long long a, long long b) {
    return eigenvalues[a] < eigenvalues[b];
  });
  std::vector<double> srt(n), w(n);
  for (long long i = 0; i < n; ++i) {
    srt[i] = eigenvalues[order[i]];
    w[i] = kw[order[i] / per_k] / (double)spin;
  }
  // sortedEnergyEigenValues / indexEnergyEigenValues (populate.F90:250-287),
  // the index 0-based here
  if (sorted_energies) std::copy(srt.begin(), srt.end(), sorted_energies);
  if (sort_index)
    for (long long i = 0; i < n; ++i) sort_index[i] = (int)order[i];
  const double ne = num_electrons;
  std::fill(population, population + n, 0.0);
  double populated = 0.0;
  long long occ = -1;
  for (long long i = 0; i < n; ++i) {
    population[order[i]] = w[i];
    populated = populated + population[order[i]];
    if (populated > ne) {
      population[order[i]] = w[i] + ne - populated;
      populated = ne;
    }
    if (std::fabs(ne - populated) < kSmallThresh) {
      occ = i;
      break;
    }
  }
  if (occ < 0) return IMAGO_ERR_RANGE;  // fewer states than electrons
  double occ_e = srt[occ];
  long long lo = occ, hi = occ;
  double degen = population[order[occ]], possible = w[occ];
  while (hi + 1 < n && std::fabs(occ_e - srt[hi + 1]) <= kSmallThresh) {
    ++hi;
    possible = possible + w[hi];
  }
  while (lo > 0 && std::fabs(occ_e - srt[lo - 1]) <= kSmallThresh) {
    --lo;
    possible = possible + w[lo];
    degen = degen + w[lo];
  }
  for (long long i = lo; i <= hi; ++i) population[order[i]] = degen / possible * w[i];
  occ = hi;
  occ_e = srt[occ];
  double gap = 0.0;
  int kind = 0;
  if (occ < n - 1) {
    gap = srt[occ + 1] - srt[occ];
    if (gap <= kMetalGapThresh) {
      gap = 0.0;
    } else {
      kind = order[occ] / per_k == order[occ + 1] / per_k ? 1 : 2;
    }
  }
  int steps = 0;
  if (thermal_sigma != 0.0) {
    double lo_e = srt[occ] - fermi_search_limit;
    double hi_e = srt[std::min(occ + 1, n - 1)] + fermi_search_limit;
    for (steps = 1; steps <= kFermiSteps; ++steps) {
      occ_e = 0.5 * (lo_e + hi_e);
      double charge = 0.0;
      std::fill(population, population + n, 0.0);
      for (long long j = 0; j < n; ++j) {
        const double f = step_function((srt[j] - occ_e) / thermal_sigma, max_thermal_range);
        if (f == 0.0) break;
        population[order[j]] = w[j] * f;
        charge = charge + population[order[j]];
      }
      if (std::fabs(charge - ne) < kSmallThresh) break;
      if (charge < ne)
        lo_e = occ_e;
      else
        hi_e = occ_e;
    }
    if (steps > kFermiSteps) steps = kFermiSteps;
  }
  info[0] = occ_e;
  info[1] = gap;
  info[2] = kind;
  info[3] = (double)occ;
  info[4] = steps;
  return IMAGO_OK;
}

extern "C" int imago_populate_states(int num_kpoints, int spin, int num_states,
                                     const double *eigenvalues,
                                     const double *kpoint_weights, double num_electrons,
                                     double thermal_sigma, double max_thermal_range,
                                     double fermi_search_limit, double *population,
                                     double *info) {
  return imago_populate_states_sorted(num_kpoints, spin, num_states, eigenvalues,
                                      kpoint_weights, num_electrons, thermal_sigma,
                                      max_thermal_range, fermi_search_limit, population,
                                      info, nullptr, nullptr);
}
