// Host set-up of the Monte Carlo tracer (see mcsetup.cpp).
#pragma once
#include <string>
#include <vector>
#include "../../include/mb3d_cu.h"
#include "devparams.h"
#include "mc.h"

namespace mb3dcu {
// LightVals of MB3D's start-up lighting with the scene's lights.
int mc_light_default(const mb3d_cu_scene &sc, mb3d_cu_mc_light &o);
// CalcParams and CalcMCT for the card: 0 or a negative status (err says why).
int mc_setup(const mb3d_cu_scene &sc, const mb3d_cu_mc_light &lv, int depth, int secant, float ssr, DevParams &p,
             McDev &m, std::string &err);
// halton_seq as 2 x 65536 words (hrx | hry << 16, hdx | hdy << 16).
const std::vector<uint32_t> &mc_halton_table();
}  // namespace mb3dcu
