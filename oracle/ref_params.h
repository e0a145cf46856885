// ref_params.h — TEST INFRASTRUCTURE: ld_params -> the reference's
// LensDiffParams (LensDiffTypes.h:128-208), shared by the checker shims.
#pragma once

#include "LensDiffTypes.h"
#include "lensdiff_b200.h"

#include <string>

// The Custom aperture's image as the checker handed it to the reference: the
// path it sits under in the reference's own aperture-image cache and the
// flags (set by ldref_set_custom_aperture in ref_shim.cpp).
struct RefCustomAperture {
    std::string path;
    bool normalize = true;
    bool invert = false;
};
inline RefCustomAperture& refCustomAperture() {
    static RefCustomAperture c;
    return c;
}

inline LensDiffParams toReference(const ld_params& p) {
    LensDiffParams r {};
    if (p.aperture_mode == LD_APERTURE_CUSTOM) {
        r.customAperturePath = refCustomAperture().path;
        r.customApertureNormalize = refCustomAperture().normalize;
        r.customApertureInvert = refCustomAperture().invert;
    }
    r.extractionMode = static_cast<LensDiffExtractionMode>(p.extraction_mode);
    r.apertureMode = static_cast<LensDiffApertureMode>(p.aperture_mode);
    r.apodizationMode = static_cast<LensDiffApodizationMode>(p.apodization_mode);
    r.spectralMode = static_cast<LensDiffSpectralMode>(p.spectral_mode);
    r.spectrumStyle = static_cast<LensDiffSpectrumStyle>(p.spectrum_style);
    r.lookMode = static_cast<LensDiffLookMode>(p.look_mode);
    r.energyMode = static_cast<LensDiffEnergyMode>(p.energy_mode);
    r.debugView = static_cast<LensDiffDebugView>(p.debug_view);
    r.inputTransfer = static_cast<LensDiffInputTransfer>(p.input_transfer);
    r.resolutionAware = p.resolution_aware != 0;
    r.threshold = p.threshold;
    r.softnessStops = p.softness_stops;
    r.pointEmphasis = p.point_emphasis;
    r.corePreserve = p.core_preserve;
    r.bladeCount = p.blade_count;
    r.roundness = p.roundness;
    r.rotationDeg = p.rotation_deg;
    r.centralObstruction = p.central_obstruction;
    r.vaneCount = p.vane_count;
    r.vaneThickness = p.vane_thickness;
    r.diffractionScalePx = p.diffraction_scale_px;
    r.pupilResolution = p.pupil_resolution;
    r.maxKernelRadiusPx = p.max_kernel_radius_px;
    r.frameShortSidePx = p.frame_short_side_px;
    r.phaseMode = static_cast<LensDiffPhaseMode>(p.phase_mode);
    r.phaseDefocus = p.phase_defocus;
    r.phaseAstigmatism0 = p.phase_astigmatism0;
    r.phaseAstigmatism45 = p.phase_astigmatism45;
    r.phaseComaX = p.phase_coma_x;
    r.phaseComaY = p.phase_coma_y;
    r.phaseSpherical = p.phase_spherical;
    r.phaseTrefoilX = p.phase_trefoil_x;
    r.phaseTrefoilY = p.phase_trefoil_y;
    r.phaseSecondaryAstigmatism0 = p.phase_secondary_astigmatism0;
    r.phaseSecondaryAstigmatism45 = p.phase_secondary_astigmatism45;
    r.phaseQuadrafoil0 = p.phase_quadrafoil0;
    r.phaseQuadrafoil45 = p.phase_quadrafoil45;
    r.phaseSecondaryComaX = p.phase_secondary_coma_x;
    r.phaseSecondaryComaY = p.phase_secondary_coma_y;
    r.pupilDecenterX = p.pupil_decenter_x;
    r.pupilDecenterY = p.pupil_decenter_y;
    r.phaseFieldStrength = p.phase_field_strength;
    r.phaseFieldEdgeBias = p.phase_field_edge_bias;
    r.phaseFieldDefocus = p.phase_field_defocus;
    r.phaseFieldAstigRadial = p.phase_field_astig_radial;
    r.phaseFieldAstigTangential = p.phase_field_astig_tangential;
    r.phaseFieldComaRadial = p.phase_field_coma_radial;
    r.phaseFieldComaTangential = p.phase_field_coma_tangential;
    r.phaseFieldSpherical = p.phase_field_spherical;
    r.phaseFieldTrefoilRadial = p.phase_field_trefoil_radial;
    r.phaseFieldTrefoilTangential = p.phase_field_trefoil_tangential;
    r.phaseFieldSecondaryAstigRadial = p.phase_field_secondary_astig_radial;
    r.phaseFieldSecondaryAstigTangential = p.phase_field_secondary_astig_tangential;
    r.phaseFieldQuadrafoilRadial = p.phase_field_quadrafoil_radial;
    r.phaseFieldQuadrafoilTangential = p.phase_field_quadrafoil_tangential;
    r.phaseFieldSecondaryComaRadial = p.phase_field_secondary_coma_radial;
    r.phaseFieldSecondaryComaTangential = p.phase_field_secondary_coma_tangential;
    r.spectrumForce = p.spectrum_force;
    r.spectrumSaturation = p.spectrum_saturation;
    r.chromaticAffectsLuma = p.chromatic_affects_luma != 0;
    r.chromaticFocus = p.chromatic_focus;
    r.chromaticSpread = p.chromatic_spread;
    r.creativeFringe = p.creative_fringe;
    r.scatterAmount = p.scatter_amount;
    r.scatterRadius = p.scatter_radius;
    r.effectGain = p.effect_gain;
    r.coreCompensation = p.core_compensation;
    r.anisotropyEmphasis = p.anisotropy_emphasis;
    r.coreGain = p.core_gain;
    r.structureGain = p.structure_gain;
    r.coreShoulder = p.core_shoulder;
    r.structureShoulder = p.structure_shoulder;
    return r;
}
