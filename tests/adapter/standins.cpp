// standins.cpp -- the out-of-line members of the stand-in reference headers
// (test infrastructure): SimulationBackend's step() overloads, restated
// from src/nemo/SimulationBackend.cpp:22-77 (prefire, the stimulus, fire,
// postfire, then the fired list), and ReadableNetwork::getSynapseSource
// (src/nemo/ReadableNetwork.cpp: the source is the high half of the id).
#include <nemo/SimulationBackend.hpp>

namespace nemo {

unsigned ReadableNetwork::getSynapseSource(const synapse_id& id) const
{
	return (unsigned) (id >> 32);
}

const Simulation::firing_output& SimulationBackend::step()
{
	prefire();
	initCurrentStimulus(0);
	finalizeCurrentStimulus(0);
	fire();
	postfire();
	return readFiring().neurons;
}

const Simulation::firing_output& SimulationBackend::step(const firing_stimulus& fstim)
{
	prefire();
	initCurrentStimulus(0);
	finalizeCurrentStimulus(0);
	setFiringStimulus(fstim);
	fire();
	postfire();
	return readFiring().neurons;
}

const Simulation::firing_output& SimulationBackend::step(const current_stimulus& istim)
{
	prefire();
	initCurrentStimulus(istim.size());
	for(const auto& s : istim) addCurrentStimulus(s.first, s.second);
	finalizeCurrentStimulus(istim.size());
	fire();
	postfire();
	return readFiring().neurons;
}

const Simulation::firing_output& SimulationBackend::step(const firing_stimulus& fstim, const current_stimulus& istim)
{
	prefire();
	initCurrentStimulus(istim.size());
	for(const auto& s : istim) addCurrentStimulus(s.first, s.second);
	finalizeCurrentStimulus(istim.size());
	setFiringStimulus(fstim);
	fire();
	postfire();
	return readFiring().neurons;
}

}
