// plugins.hpp -- neuron types from their .ini descriptors (the role of
// nemo::NeuronType and nemo::Plugin's search path, src/nemo/NeuronType.cpp,
// src/nemo/Plugin.cpp).
#pragma once

#include <string>

#include "common.hpp"

namespace nemo_b200 {

// nemo_add_plugin_path: a directory searched for descriptors before the
// user's and the library's plugin directories (NEMO_DL_ERROR if it does not
// exist)
void addPluginPath(const std::string& dir);

// the library's own plugin directory: plugins/ beside the directory of
// libnemo_b200.so
std::string systemPluginDirectory();

// the descriptor file of a type (NEMO_INVALID_INPUT if none is found)
std::string pluginConfigurationFile(const std::string& name);

// the type described by <name>.ini, with the kernel of this backend that
// implements it (KIND_NONE if none); NEMO_INVALID_INPUT for a malformed or
// incomplete descriptor, NEMO_IO_ERROR if it cannot be read
NeuronTypeDesc parseNeuronType(const std::string& name);

// NEMO_DL_ERROR unless the backend has a kernel for the type whose layout
// matches the descriptor (simulation creation)
void checkKernelBinding(const NeuronTypeDesc& d);

} // namespace nemo_b200
