"""Neuron types from .ini descriptors (src/nemo/NeuronType.cpp:45-156,
src/nemo/Plugin.cpp:185-195): the search order (directories added with
nemo_add_plugin_path, then ~/.nemo/plugins, then the library's own
plugins/ directory), the descriptor keys, the errors of a missing or
malformed descriptor, and the binding of a type to a kernel of this backend
when a simulation is created.  CPU only: nothing here launches a kernel
(simulation creation fails before it touches a device)."""
import os

import numpy as np
import pytest

import nemosim_b200 as nb

NEMO_INVALID_INPUT, NEMO_DL_ERROR = 6, 12


def descriptor(params=1, state=1, mpot=0, normal="false", extra=""):
    return (f"# a test type\nparameters={params}\nstate-variables={state}\nmembrane-potential={mpot}\n"
            f"history=1\n\n[rcm]\nsources=false\n\n[rng]\nnormal={normal}\n\n[backends]\ncuda=true\n{extra}")


def write(directory, name, text):
    os.makedirs(directory, exist_ok=True)
    with open(os.path.join(directory, name + ".ini"), "w") as f:
        f.write(text)


@pytest.fixture
def home(tmp_path, monkeypatch):
    """A fresh home directory, so ~/.nemo/plugins is empty unless a test
    fills it (the search reads HOME at each lookup)."""
    h = tmp_path / "home"
    h.mkdir()
    monkeypatch.setenv("HOME", str(h))
    return h


def args_accepted(ntype_name, nargs):
    net = nb.Network()
    t = net.add_neuron_type(ntype_name)
    try:
        net.add_neuron(t, 0, *([0.0] * nargs))
        return True
    except nb.NemoError as e:
        assert e.code == NEMO_INVALID_INPUT
        return False


def test_shipped_descriptors(home):
    """The library's descriptors give the reference's layouts."""
    for name, nargs in [("Izhikevich", 7), ("IF_curr_exp", 13), ("PoissonSource", 1), ("Input", 0),
                        ("IzhikevichRS", 2), ("Kuramoto", 2)]:
        assert args_accepted(name, nargs), name
        assert not args_accepted(name, nargs + 1), name


def test_user_directory_before_library_directory(home):
    write(home / ".nemo" / "plugins", "Izhikevich", descriptor(params=6, state=2, mpot=1, normal="true"))
    assert args_accepted("Izhikevich", 8)
    assert not args_accepted("Izhikevich", 7)


def test_added_path_before_user_directory(home, tmp_path):
    write(home / ".nemo" / "plugins", "OrderProbeA", descriptor(params=2))
    extra = tmp_path / "extra"
    write(extra, "OrderProbeA", descriptor(params=3))
    assert args_accepted("OrderProbeA", 3)  # not yet added: the user's
    nb.add_plugin_path(str(extra))
    assert args_accepted("OrderProbeA", 4)
    assert not args_accepted("OrderProbeA", 3)


def test_added_paths_are_searched_in_order(home, tmp_path):
    """Added directories form an ordered set (the reference keeps them in a
    std::set of paths), searched in that order."""
    a, b = tmp_path / "a_dir", tmp_path / "b_dir"
    write(a, "OrderProbeB", descriptor(params=5))
    write(b, "OrderProbeB", descriptor(params=7))
    nb.add_plugin_path(str(b))
    nb.add_plugin_path(str(a))
    nb.add_plugin_path(str(a))  # a repeat changes nothing
    assert args_accepted("OrderProbeB", 6)


def test_missing_plugin_path_fails():
    with pytest.raises(nb.NemoError) as e:
        nb.add_plugin_path("/nonexistent/plugin/dir")
    assert e.value.code == NEMO_DL_ERROR


def test_unknown_type_fails(home):
    with pytest.raises(nb.NemoError) as e:
        nb.Network().add_neuron_type("NoSuchNeuronType")
    assert e.value.code == NEMO_INVALID_INPUT


@pytest.mark.parametrize("text,what", [
    (descriptor(extra="colour=blue\n"), "unknown key"),
    (descriptor(normal="maybe"), "bad bool"),
    ("parameters=1\nstate-variables=1\nmembrane-potential=0\n", "missing rng.normal"),
    ("state-variables=1\nmembrane-potential=0\n[rng]\nnormal=false\n", "missing parameters"),
    (descriptor(params="-1"), "negative count"),
    (descriptor(extra="history=2\n"), "repeated key"),
    (descriptor(extra="just words\n"), "line without '='"),
])
def test_malformed_descriptor_fails(home, text, what):
    write(home / ".nemo" / "plugins", "BadProbe", text)
    with pytest.raises(nb.NemoError) as e:
        nb.Network().add_neuron_type("BadProbe")
    assert e.value.code == NEMO_INVALID_INPUT, what


def test_comments_sections_and_bool_spellings(home):
    text = ("# comment line\n  parameters = 2   # trailing comment\nstate-variables=0\nmembrane-potential=0\n"
            "[rng]\nnormal = Off\n[rcm]\nweights=yes\n[backends]\ncpu=0\ncuda=On\n")
    write(home / ".nemo" / "plugins", "SpellingProbe", text)
    assert args_accepted("SpellingProbe", 2)


def test_invalid_type_index():
    """testInvalidNeuronType (src/test/test.cpp:966-978): an index that is
    not a type of the network fails."""
    net = nb.Network()
    iz = net.add_neuron_type("Izhikevich")
    for n in range(1, 20):
        with pytest.raises(nb.NemoError):
            net.add_neuron(n, iz, *([0.0] * 7))


def test_type_without_kernel_fails_at_simulation_creation(home):
    """A type the backend has no kernel for is accepted by the network and
    fails when a simulation is created, as the reference fails to load the
    type's backend plugin (NEMO_DL_ERROR)."""
    write(home / ".nemo" / "plugins", "NoKernelProbe", descriptor(params=1, state=1))
    net = nb.Network()
    t = net.add_neuron_type("NoKernelProbe")
    net.add_neuron(t, 0, 1.0, 2.0)
    with pytest.raises(nb.NemoError) as e:
        nb.Simulation(net, nb.Configuration())
    assert e.value.code == NEMO_DL_ERROR


def test_layout_mismatch_fails_at_simulation_creation(home):
    """A descriptor that gives a compiled type another layout than its
    kernel's is rejected when a simulation is created."""
    write(home / ".nemo" / "plugins", "Izhikevich", descriptor(params=6, state=2, mpot=1, normal="true"))
    net = nb.Network()
    t = net.add_neuron_type("Izhikevich")
    net.add_neuron(t, 0, *([0.0] * 8))
    with pytest.raises(nb.NemoError) as e:
        nb.Simulation(net, nb.Configuration())
    assert e.value.code == NEMO_DL_ERROR
