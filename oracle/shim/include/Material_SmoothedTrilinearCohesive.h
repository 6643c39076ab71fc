/* Declaration of TrilinearSmoothedCohesiveMaterial for the oracle build of the reference (test
 * infrastructure only; the reference ships src/Material_SmoothedTrilinearCohesive.cpp without
 * this header).  Declared from the members that .cpp defines, on top of the no-unloading smoothed
 * class.  One internal variable per point: the maximum opening. */
#pragma once
#include "Material_SmoothedTrilinearCohesiveNU.h"

class TrilinearSmoothedCohesiveMaterial : public TrilinearSmoothedCohesiveNUMaterial {
 public:
  virtual ~TrilinearSmoothedCohesiveMaterial() {}
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
