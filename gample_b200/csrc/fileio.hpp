// fileio.hpp -- the reference's binary outputs and restart files
// (src/FileIO.{h,mm}); paths are relative to the working directory, under
// bin/, with the reference's names and byte layouts:
//   bin/<Project>_EMField_%08d.bin          header ngx, ngy, ngb (int32), dx, dy
//   bin/<Project>_Moments_<name>_%08d.bin   (float32), then records of a
//                                           32-byte name, an int32 type id and
//                                           the scaled float32 array
//   bin/<Project>_PhaseSpace_<name>_<k>.bin appended (cycle, x, y, vx, vy, vz)
//                                           of particles k = 0..19
//   bin/<Project>_ProgressData_<name>_%08d.bin  pNum 24-byte particle records
#pragma once

#include <string>
#include <vector>

#include "pic.hpp"

namespace gample {

void outputField(int cycle, EMField& fld, const Init& init, XmlLogger* logger);                  // :41-136
void outputMoments(int cycle, Moment& mom, const std::string& pName, const Init& init, XmlLogger* logger);  // :138-226
void outputPhaseSpace(int cycle, Particle& p, const Init& init);                                  // :4-39
bool saveProgress(int cycle, std::vector<Particle*>& ptcls, const Init& init);                    // :250-293
bool loadProgress(int cycle, std::vector<Particle*>& ptcls, const Init& init);                    // :295-352

}  // namespace gample
