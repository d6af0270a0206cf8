"""A cellweave configuration file read as SimConfig does (crates/io/src/config.rs), on CPU."""
import os

import numpy as np
import pytest

import cellweave_b200 as cw
from cellweave_b200 import config as C

NET = """
[[nodes]]
name = "a"
initial = 0.5
terms = [ { kind = "activated_by", source = "oxygen", rate = 0.5 }, { kind = "decays", rate = 0.3 } ]
[roles]
growth = "a"
survival = "a"
hypoxia_response = "a"
[mechanics]
growth_coefficient = 0.5
lambda_volume = 40.0
"""


def write(tmp_path, text, net=True):
    if net:
        (tmp_path / "net.toml").write_text(NET)
    p = tmp_path / "run.toml"
    p.write_text(text)
    return str(p)


BASE = """width = 60
height = 50
mcs = 30
temperature = 10.0
snapshot_interval = 10
output_dir = "out"
network = "net.toml"
"""


def test_defaults_are_the_reference_configurations(tmp_path):
    cfg = C.load_sim_config(write(tmp_path, BASE))
    # config.rs:12-140 with its serde defaults
    assert cfg["depth"] == 1 and cfg["max_cells"] == 2000 and cfg["seed"] == 42
    assert cfg["oxygen_source"] == {"kind": "bath"} and cfg["seeding"] == {"kind": "single"}
    assert cfg["oxygen_uptake"] == 0.00002 and cfg["sweeps_per_step"] == 1 and cfg["contact_order"] == 1
    assert cfg["network_path"] == os.path.join(str(tmp_path), "net.toml")
    kw, refvol = C.simulation_kwargs(cfg)
    # one disc of radius 8 at the centre: 197 pixels, the network's reference volume
    assert refvol == 197
    assert kw["o2_hold"] == 3 and kw["seeding"] == 3 and kw["seed_side"] == 8 and kw["divide_every"] == 20
    assert kw["o2_dcoef"] == 0.2 and kw["dt"] == 1.0 and kw["substeps"] == 8 and kw["necrotic_type"] == 3
    np.testing.assert_array_equal(C.CONTACT, C.CONTACT.T)


def test_a_vessel_seeds_its_cell_against_the_wall(tmp_path):
    cfg = C.load_sim_config(write(tmp_path, BASE + "\n[oxygen_source]\nkind = \"vessel\"\nradius = 6\n"))
    kw, refvol = C.simulation_kwargs(cfg)
    assert kw["o2_hold"] == 4 and kw["vessel_radius"] == 6
    # the ball's centre is radius + 8 from the vessel's: their edges meet on one
    # pixel, which stays vessel (add_ball skips obstacles, cpm.rs:338-339)
    assert refvol == 196


def test_what_the_device_step_does_not_run_is_refused_by_name(tmp_path):
    for extra, word in [("\n[oxygen_source]\nkind = \"capillary\"\nradius = 3\n", "capillary"),
                        ("\n[seeding]\nkind = \"sheet\"\nside = 10\n", "sheet"),
                        ("mutation_rate = 1.5\n", "mutation_rate"),
                        ("suppress = [1]\n", "suppress"),
                        ("\n[angiogenesis]\nthreshold = 0.5\n", "angiogenesis"),
                        ("\n[lesion]\nat = 10\nradius = 4\n", "lesion"),
                        ("contact_order = 4\n", "contact_order")]:
        cfg = C.load_sim_config(write(tmp_path, (extra + BASE) if extra.startswith("\n") is False else BASE + extra))
        with pytest.raises(cw.ConfigError, match=word):
            C.simulation_kwargs(cfg)
    with pytest.raises(cw.ConfigError, match="mcs"):
        C.load_sim_config(write(tmp_path, BASE.replace("mcs = 30\n", "")))
    with pytest.raises(cw.ConfigError, match="network"):
        C.simulation_kwargs(C.load_sim_config(write(tmp_path, BASE.replace('network = "net.toml"\n', ""))))


def test_mutation_and_rewiring_map_onto_the_step(tmp_path):
    cfg = C.load_sim_config(write(tmp_path, "mutation_rate = 0.05\nrewiring = 0.3\n" + BASE))
    kw, _ = C.simulation_kwargs(cfg)
    assert kw["mutation_rate"] == 0.05 and kw["rewiring"] == 0.3
    kw, _ = C.simulation_kwargs(C.load_sim_config(write(tmp_path, BASE)))
    assert "mutation_rate" not in kw


def test_a_lesion_and_suppressed_mutations_are_read_and_checked(tmp_path):
    # LesionConfig (config.rs:142-160) and the checks of simulation.rs:751-770
    sheet = BASE + "oxygen_uptake = 0.0\nmutation_rate = 0.01\nsuppress_before = 40\n[seeding]\nkind = \"sheet\"\nside = 10\n"
    cfg = C.load_sim_config(write(tmp_path, sheet + "[lesion]\nnetwork = \"net.toml\"\nat = 20\nradius = 15.0\n"))
    kw, refvol = C.simulation_kwargs(cfg)
    assert kw["suppress_before"] == 40 and refvol == 100 and cfg["lesion"]["at"] == 20
    for lesion, word in [("at = 20\nradius = 15.0\n", "network"),
                         ("network = \"net.toml\"\nat = 20\nradius = 0.0\n", "radius"),
                         ("network = \"net.toml\"\nat = 20\nradius = 5.0\ncentre = [60.0, 10.0]\n", "outside")]:
        cfg = C.load_sim_config(write(tmp_path, sheet + "[lesion]\n" + lesion))
        with pytest.raises(cw.ConfigError, match=word):
            C.simulation_kwargs(cfg)
    vol = BASE.replace("height = 50\n", "height = 50\ndepth = 20\n") + "[lesion]\nnetwork = \"net.toml\"\nat = 2\nradius = 3.0\n"
    with pytest.raises(cw.ConfigError, match="plane"):
        C.simulation_kwargs(C.load_sim_config(write(tmp_path, vol)))


def test_tracing_is_read_and_checked(tmp_path):
    # Tracing (types.rs:208-214) and its check (simulation.rs:614-619)
    sheet = BASE + "oxygen_uptake = 0.0\n[seeding]\nkind = \"sheet\"\nside = 10\n"
    kw, _ = C.simulation_kwargs(C.load_sim_config(write(tmp_path, sheet + "[tracing]\nat = 30\nevery = 10\n")))
    assert kw["tracing_at"] == 30
    with pytest.raises(cw.ConfigError, match="every 0 steps"):
        C.simulation_kwargs(C.load_sim_config(write(tmp_path, sheet + "[tracing]\nat = 30\nevery = 0\n")))
    with pytest.raises(cw.ConfigError, match="every"):
        C.simulation_kwargs(C.load_sim_config(write(tmp_path, sheet + "[tracing]\nat = 30\n")))


def test_released_fields_map_onto_the_step(tmp_path):
    cfg = C.load_sim_config(write(tmp_path, BASE + "\n[waste]\nproduction = 0.01\n[necrotic_factor]\n"
                                                   "production = 0.05\nrelease_for = 12\n"))
    kw, _ = C.simulation_kwargs(cfg)
    assert kw["waste_production"] == 0.01 and kw["necrotic_production"] == 0.05 and kw["necrotic_release_for"] == 12


def test_the_edge_is_the_boxs_sides_and_a_baths_faces():
    g = np.zeros((1, 10, 10), np.int32)
    g[0, 4:6, 4:6] = 1
    assert not C.touches_the_edge(g)
    g[0, 0, 5] = 1
    assert C.touches_the_edge(g)
    v = np.zeros((5, 10, 10), np.int32)
    v[0, 5, 5] = 1
    assert C.touches_the_edge(v) and not C.touches_the_edge(v, vessel=True)


def test_a_cycle_of_its_own_divides_every_step_and_is_checked(tmp_path):
    cfg = C.load_sim_config(write(tmp_path, BASE + "\n[cycle]\nmedian = 20.0\nspread = 0.3\n"))
    kw, _ = C.simulation_kwargs(cfg)
    # divide_ready_cells every step with a cycle (simulation.rs:1341-1344)
    assert kw["cycle_median"] == 20.0 and kw["cycle_spread"] == 0.3 and kw["divide_every"] == 1
    # the first solve is start()'s (simulation.rs:91-98)
    assert kw["first_tolerance"] == 1e-8
    with pytest.raises(cw.ConfigError, match="median and its spread"):
        C.simulation_kwargs(C.load_sim_config(write(tmp_path, BASE + "\n[cycle]\nmedian = 20.0\n")))
    plain, _ = C.simulation_kwargs(C.load_sim_config(write(tmp_path, BASE)))
    assert "cycle_median" not in plain and plain["divide_every"] == 20


def test_debris_loss_and_a_still_medium_are_carried(tmp_path):
    cfg = C.load_sim_config(write(tmp_path, "depth = 40\ndebris_loss = 0.024\n" + BASE.replace("width = 60", "width = 40")
                                  .replace("height = 50", "height = 40") + "\n[still_medium]\ndiffusion = 0.606\n"))
    kw, refvol = C.simulation_kwargs(cfg)
    assert kw["debris_loss"] == 0.024 and kw["still_medium"] == 0.606
    # a ball of radius 3 in a volume (simulation.rs:74)
    assert kw["seed_side"] == 3 and refvol == 123


def test_an_exposure_is_read_with_its_schedule(tmp_path):
    per = "\n[exposure]\nintensity = 0.8\nuptake = 0.001\nstart = 100\nschedule = { kind = \"periodic\", on = 5, off = 7 }\n"
    kw, _ = C.simulation_kwargs(C.load_sim_config(write(tmp_path, BASE + per)))
    assert (kw["exposure_intensity"], kw["exposure_uptake"], kw["exposure_start"]) == (0.8, 0.001, 100)
    assert (kw["exposure_on"], kw["exposure_off"]) == (5, 7)
    cont = per.replace('{ kind = "periodic", on = 5, off = 7 }', '{ kind = "continuous" }')
    kw, _ = C.simulation_kwargs(C.load_sim_config(write(tmp_path, BASE + cont)))
    assert (kw["exposure_on"], kw["exposure_off"]) == (0, 0)
    never = per.replace("on = 5", "on = 0")
    with pytest.raises(cw.ConfigError, match="never on"):
        C.simulation_kwargs(C.load_sim_config(write(tmp_path, BASE + never)))
    with pytest.raises(cw.ConfigError, match="uptake"):
        C.simulation_kwargs(C.load_sim_config(write(tmp_path, BASE + per.replace("uptake = 0.001\n", ""))))


def test_the_runner_refuses_a_configuration_it_cannot_run(tmp_path, capsys):
    path = write(tmp_path, BASE + "\n[lesion]\nat = 3\nradius = 2\n")
    with pytest.raises(cw.ConfigError, match="lesion"):
        C.main([path, "--steps", "2"])


def test_the_example_shaped_scenarios_load(tmp_path):
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "make_scenarios", os.path.join(os.path.dirname(__file__), "golden", "make_scenarios.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.main(str(tmp_path))
    for name in mod.SCENARIOS:
        kw, refvol = C.simulation_kwargs(C.load_sim_config(str(tmp_path / f"{name}.toml")))
        assert refvol > 0 and kw["first_tolerance"] == 1e-8
    kw, _ = C.simulation_kwargs(C.load_sim_config(str(tmp_path / "spheroid3d.toml")))
    assert kw["debris_loss"] == 0.024 and kw["still_medium"] == 0.606 and kw["cycle_median"] == 20.0
    assert kw["dims"] == [(320, 320, 320)] and kw["max_cells"] == 200000 and kw["sweeps"] == 4


# crates/io/src/config.rs:702-866: a network file and the chain it extends
EXT_BASE = ('[[nodes]]\nname = "a"\ninitial = 0.1\nterms = [ { kind = "decays", rate = 0.5 } ]\n\n'
            '[[nodes]]\nname = "b"\ninitial = 0.2\n\n'
            '[roles]\ngrowth = "a"\nsurvival = "b"\nhypoxia_response = "b"\n\n'
            '[mechanics]\ngrowth_coefficient = 1.0\nlambda_volume = 2.0\n')


def test_extending_replaces_a_node_whole_appends_new_ones_and_inherits_the_rest(tmp_path):
    (tmp_path / "base.toml").write_text(EXT_BASE)
    (tmp_path / "child.toml").write_text('extends = "base.toml"\n\n[[nodes]]\nname = "a"\ninitial = 0.9\nterms = []\n')
    spec = cw.load_network_spec(str(tmp_path / "child.toml"))
    assert [n["name"] for n in spec["nodes"]] == ["a", "b"]
    assert spec["nodes"][0]["initial"] == 0.9 and spec["nodes"][0]["terms"] == []
    assert spec["nodes"][1]["initial"] == 0.2
    assert spec["roles"]["survival"] == "b" and spec["mechanics"]["lambda_volume"] == 2.0
    assert spec.get("extends") is None
    (tmp_path / "more.toml").write_text('extends = "base.toml"\n\n[[nodes]]\nname = "c"\ninitial = 0.3\n')
    assert [n["name"] for n in cw.load_network_spec(str(tmp_path / "more.toml"))["nodes"]] == ["a", "b", "c"]


def test_a_chain_of_three_is_laid_youngest_over_oldest(tmp_path):
    (tmp_path / "base.toml").write_text(EXT_BASE)
    (tmp_path / "middle.toml").write_text('extends = "base.toml"\n\n[[nodes]]\nname = "a"\ninitial = 0.5\n')
    (tmp_path / "top.toml").write_text('extends = "middle.toml"\n\n[[nodes]]\nname = "b"\ninitial = 0.7\n')
    spec = cw.load_network_spec(str(tmp_path / "top.toml"))
    assert spec["nodes"][0]["initial"] == 0.5 and spec["nodes"][1]["initial"] == 0.7


def test_a_loop_and_a_contact_energy_in_a_network_are_refused(tmp_path):
    (tmp_path / "one.toml").write_text('extends = "two.toml"\n')
    (tmp_path / "two.toml").write_text('extends = "one.toml"\n')
    with pytest.raises(cw.ConfigError, match="loop") as e:
        cw.load_network_spec(str(tmp_path / "one.toml"))
    assert "one.toml" in str(e.value) and "two.toml" in str(e.value)
    (tmp_path / "base.toml").write_text(EXT_BASE)
    (tmp_path / "sticky.toml").write_text('extends = "base.toml"\n\n[mechanics]\ngrowth_coefficient = 1.0\n'
                                          'lambda_volume = 2.0\nj_medium = 16.0\n')
    with pytest.raises(cw.ConfigError, match="j_medium"):
        cw.load_network_spec(str(tmp_path / "sticky.toml"))
    (tmp_path / "lonely.toml").write_text('[[nodes]]\nname = "a"\n')
    lonely = cw.load_network_spec(str(tmp_path / "lonely.toml"))
    assert lonely.get("roles") is None and lonely.get("mechanics") is None
    with pytest.raises(cw.ConfigError, match="no roles"):
        cw.Network.from_spec(lonely, 100)


def test_the_shipped_mutant_differs_from_its_base_in_one_node(golden):
    # config.rs:866-898 on the networks the fixtures carry
    mutant, base = golden["networks"]["ras-erk-mutant"], golden["networks"]["ras-erk"]
    assert len(mutant["nodes"]) == len(base["nodes"])
    assert [m["name"] for m, b in zip(mutant["nodes"], base["nodes"]) if m != b] == ["ras"]
    assert mutant["roles"] == base["roles"] and mutant["mechanics"] == base["mechanics"]


def test_a_missing_network_file_is_reported_with_its_path(tmp_path):
    # config.rs:681-692
    with pytest.raises(cw.ConfigError, match="nowhere/at/all.toml"):
        cw.load_network_spec(str(tmp_path / "nowhere" / "at" / "all.toml"))
    cfg = C.load_sim_config(write(tmp_path, BASE.replace('"net.toml"', '"nowhere/at/all.toml"'), net=False))
    with pytest.raises(cw.ConfigError, match="nowhere/at/all.toml"):
        cw.load_network_spec(cfg["network_path"])


def test_a_cycle_lasts_a_step_at_least_and_spreads_by_something(tmp_path):
    # simulation.rs:2849-2866
    for median, spread in [("0.5", "0.2"), ("20.0", "-0.1"), ("nan", "0.2"), ("20.0", "inf")]:
        text = BASE + f"\n[cycle]\nmedian = {median}\nspread = {spread}\n"
        with pytest.raises(cw.ConfigError, match="a cycle lasts a step at least"):
            C.simulation_kwargs(C.load_sim_config(write(tmp_path, text)))


def test_the_oracles_cycle_lengths_have_the_median_and_spread_asked_for():
    # simulation.rs:2868-2888: 4000 draws of median 40, spread 0.3
    from oracle import cpu_sim
    hist = cpu_sim.CpuHistory.__new__(cpu_sim.CpuHistory)
    hist.cfg, hist.div_rng = {"cycle_median": 40.0, "cycle_spread": 0.3}, np.random.default_rng(7)
    logs = np.sort(np.log([hist._cycle_length() for _ in range(4000)]))
    assert abs(np.exp(logs[len(logs) // 2]) - 40.0) < 2.0
    assert abs(logs.std() - 0.3) < 0.03


def test_a_debris_loss_is_a_share_per_step_and_a_step_sweeps_at_least_once(tmp_path):
    # simulation.rs:3085-3103
    for loss in ("0.0", "-0.1", "1.5", "nan"):
        with pytest.raises(cw.ConfigError, match="debris loss"):
            C.simulation_kwargs(C.load_sim_config(write(tmp_path, f"debris_loss = {loss}\n" + BASE)))
    with pytest.raises(cw.ConfigError, match="at least once"):
        C.simulation_kwargs(C.load_sim_config(write(tmp_path, "sweeps_per_step = 0\n" + BASE)))


def test_a_ceiling_below_the_division_ratio_is_refused(tmp_path):
    # simulation.rs:3416-3423 (the check, 621-628), before anything reaches the device
    path = write(tmp_path, BASE)
    (tmp_path / "net.toml").write_text(NET + "max_target = 1.2\n")
    with pytest.raises(cw.ConfigError, match="no cell could ever divide"):
        C.simulation_from_config(C.load_sim_config(path))
