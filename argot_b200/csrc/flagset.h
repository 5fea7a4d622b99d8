// flagset.h -- the reference's compile-time flag set as this library sees it.
//
// ARGOT selects its chemistry and its rate formula with preprocessor flags
// (src/Makefile:149-196): __HELIUM__ adds HeI/HeII columns and rates,
// __HYDROGEN_MOL__ adds H-, H2 and H2+ columns and rates (src/radiation.h,
// src/prim_chem/chemistry.h:41-63), __PHOTON_CONSERVING__ selects the
// photon-conserving cell factor (src/calc_photoion_rate.c:327-386, else
// :291-326) and __COSMOLOGICAL__ scales columns and distances by the scale
// factor (:260-276).  The struct layouts that cross the drop-in boundary
// follow the first two.  The library is compiled once per flag set with the
// caller's own flags (argot_b200/build.py: the default set and the stock
// set of src/Makefile, plus the other combinations the tests cover); without
// ARGOT_FLAGSET_EXPLICIT it takes the default set below.
#pragma once

#ifndef ARGOT_FLAGSET_EXPLICIT
// the library's default: helium, photon conserving, no H2, not cosmological
#ifndef __HELIUM__
#define __HELIUM__
#endif
#ifndef __PHOTON_CONSERVING__
#define __PHOTON_CONSERVING__
#endif
#endif

// Entry points tied to one layout: the ART drop-in and the device API's
// packing of a struct fluid_mesh array read the helium fields of the
// default layout (and ART's own scale-factor terms are not carried).
#if defined(__HELIUM__) && !defined(__HYDROGEN_MOL__) && !defined(__COSMOLOGICAL__)
#define ARGOT_HELIUM_LAYOUT 1
#endif

namespace argot {
namespace flags {

#ifdef __HELIUM__
constexpr bool kHe = true;
#else
constexpr bool kHe = false;
#endif
#ifdef __HYDROGEN_MOL__
constexpr bool kH2 = true;
#else
constexpr bool kH2 = false;
#endif
#ifdef __PHOTON_CONSERVING__
constexpr bool kPC = true;
#else
constexpr bool kPC = false;
#endif
#ifdef __COSMOLOGICAL__
constexpr bool kCosmo = true;
#else
constexpr bool kCosmo = false;
#endif

// The set the device-resident fast path computes (three columns, the
// photon-conserving rates, no scale factor).
constexpr bool kDefault = kHe && !kH2 && kPC && !kCosmo;

// Columns per segment and per ray, in the reference's field order:
// HI, [HeI, HeII], [HM, H2I, H2II].
constexpr int kNCol = 1 + (kHe ? 2 : 0) + (kH2 ? 3 : 0);
constexpr int kColHeI = 1, kColHeII = 2;
constexpr int kColHM = kHe ? 3 : 1, kColH2I = kColHM + 1, kColH2II = kColHM + 2;

// Cross-section channels of struct cross_section (src/cross_section.h:7-20):
// HI, [HeI, HeII], [HM, H2I_I, H2II_I, H2II_II].
constexpr int kNChan = 1 + (kHe ? 2 : 0) + (kH2 ? 4 : 0);

// Rate fields of struct prim_chem from GammaHI on, in its order:
// GammaHI, HeatHI, [GammaHeI, GammaHeII, HeatHeI, HeatHeII],
// [GammaHM, GammaH2I_I, GammaH2I_II, GammaH2II_I, GammaH2II_II,
//  HeatHM, HeatH2I_I, HeatH2I_II, HeatH2II_I, HeatH2II_II].
constexpr int kNOut = 2 + (kHe ? 4 : 0) + (kH2 ? 10 : 0);
constexpr int kOutGHI = 0, kOutHHI = 1;
constexpr int kOutGHeI = 2, kOutGHeII = 3, kOutHHeI = 4, kOutHHeII = 5;
constexpr int kOutH2 = kHe ? 6 : 2;  // GammaHM
constexpr int kOutGHM = kOutH2, kOutGH2I_I = kOutH2 + 1, kOutGH2I_II = kOutH2 + 2, kOutGH2II_I = kOutH2 + 3,
              kOutGH2II_II = kOutH2 + 4;
constexpr int kOutHHM = kOutH2 + 5, kOutHH2I_I = kOutH2 + 6, kOutHH2I_II = kOutH2 + 7, kOutHH2II_I = kOutH2 + 8,
              kOutHH2II_II = kOutH2 + 9;

// Name of the flag set (argot_b200_flagset()).
constexpr const char *kName =
    kHe ? (kH2 ? (kPC ? (kCosmo ? "helium+h2, photon conserving, cosmological" : "helium+h2, photon conserving")
                      : (kCosmo ? "helium+h2, cosmological" : "helium+h2"))
               : (kPC ? (kCosmo ? "helium, photon conserving, cosmological" : "helium, photon conserving")
                      : (kCosmo ? "helium, cosmological" : "helium")))
        : (kH2 ? (kPC ? (kCosmo ? "h2, photon conserving, cosmological" : "h2, photon conserving")
                      : (kCosmo ? "h2, cosmological" : "h2"))
               : (kPC ? (kCosmo ? "hydrogen, photon conserving, cosmological" : "hydrogen, photon conserving")
                      : (kCosmo ? "hydrogen, cosmological" : "hydrogen")));

}  // namespace flags
}  // namespace argot
