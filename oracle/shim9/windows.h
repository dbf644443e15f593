/*
 * Empty stand-in for <windows.h>.  TEST INFRASTRUCTURE ONLY: the reference's
 * Homogenization/QNC/mgcg9.cu includes it (a Windows MEX build) but uses
 * nothing from it on the solver path; this lets the unmodified source
 * compile on Linux for the oracle's reference build.
 */
#pragma once
