/* Declaration of TrilinearCohesiveMaterial for the oracle build of the reference (test
 * infrastructure only).  The reference ships src/Material_TrilinearCohesive.cpp without this
 * header; the class is declared here from the members that .cpp defines, on top of the
 * no-unloading class whose header the reference does ship (the same layering as its bilinear
 * pair).  One internal variable per point: the maximum opening. */
#pragma once
#include "Material_TrilinearCohesiveNU.h"

class TrilinearCohesiveMaterial : public TrilinearCohesiveNUMaterial {
 public:
  virtual ~TrilinearCohesiveMaterial() {}
  virtual Material* allocate();
  virtual material_type get_type() { return TL_COHESIVE; }
  virtual Material::output_params* Constitutive(Material::input_params& input);
  virtual id_type n_internal_vars() { return 1; }
  virtual std::vector<double> init_internal_vars() { return std::vector<double>(1, 0.0); }
  virtual std::vector<double> max_internal_vars() { return std::vector<double>(1, 1.0); }
  virtual std::vector<std::string> internal_vars_name();
  virtual std::vector<bool> internal_vars_print();
  virtual Material::sensitivity_output_params* SensitivityConstitutive(Material::sensitivity_input_params& input);
  virtual void updateSensitivityISVs(Material::sensitivity_input_params& input);
};
