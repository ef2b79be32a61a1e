// Link stubs for the oracle harness (test infrastructure only).
//
// SORT's mesh, visual and accelerator objects reference material, medium and
// 3D-texture code that needs the absent TSL library. None of it is reached on
// the ray-query path the harness drives (opaque materials, no media, no
// volume textures), so these definitions only satisfy the linker. Each one
// returns a neutral value.
#include "material/material.h"
#include "material/matmanager.h"
#include "medium/medium.h"
#include "medium/mediumdata.h"
#include "texture/imagetexture3d.h"

void Material::UpdateScatteringEvent(ScatteringEvent&, RenderContext&) const {}
void Material::UpdateMediumStack(const MediumInteraction&, const SE_Interaction, MediumStack&, RenderContext&) const {}
void Material::EvaluateMediumSample(const MediumInteraction&, MediumSample&) const {}
void Material::Serialize(IStreamBase&) {}
void Material::BuildMaterial(Tsl_Namespace::ShadingContext*) {}

const MaterialBase* MatManager::CreateMaterialProxy(const MaterialBase& material) { return &material; }


float MediumDensity::Sample(const Point&) const { return 0.0f; }
void MediumDensity::Serialize(IStreamBase&) {}
Spectrum MediumColor::Sample(const Point&) const { return 0.0f; }
void MediumColor::Serialize(IStreamBase&) {}

template <> float ImageTexture3D<float>::Sample(int, int, int) const { return 0.0f; }
template <> float ImageTexture3D<float>::Sample(float, float, float) const { return 0.0f; }
template <> Spectrum ImageTexture3D<Spectrum>::Sample(int, int, int) const { return 0.0f; }
template <> Spectrum ImageTexture3D<Spectrum>::Sample(float, float, float) const { return 0.0f; }
