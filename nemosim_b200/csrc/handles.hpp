// handles.hpp -- the objects behind the C ABI's opaque handles.
#pragma once

#include <memory>

#include "bptt.hpp"
#include "network.hpp"
#include "simulation.hpp"

struct nemo_network_class { nemo_b200::Network net; };
struct nemo_configuration_class { nemo_b200::Configuration conf; };
struct nemo_simulation_class { std::unique_ptr<nemo_b200::Simulation> sim; };
struct nemo_b200_bptt_class { std::unique_ptr<nemo_b200::Bptt> impl; };
