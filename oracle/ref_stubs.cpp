/*
 * Definitions for the five solver entry points that GO-Ferro's public
 * sources declare but never define (ferroelectric_system.h:103-106,
 * elastic_system.h:190-199).  Without them the reference does not link.
 *
 * TEST INFRASTRUCTURE for the CPU oracle only.
 *
 * Each is a no-op: the static fields they would fill (Ex_stat..., exxt0_*...)
 * stay at the zeros matrix3d::initialize gives them (matrix.h:18-25), unless
 * the deck loads them from Estat.in / strain files.  Decks used for parity
 * therefore keep the electrostatic and elastostatic solvers out of the
 * compared physics.
 */
#include "ferroelectric_system.h"
#include "elastic_system.h"

void ferroelectric_system::get_E_static() {}
void ferroelectric_system::get_E_static_1D() {}
void elastic_system::get_strain_static() {}
void elastic_system::get_strain_static_glb() {}
void elastic_system::get_strain_static_glb_gradient() {}
