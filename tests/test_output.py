"""measurements.csv as the reference writes it (crates/io/src/output.rs), on CPU."""
from cellweave_b200.output import MEASUREMENT_COLUMNS, MeasurementLog, measurement_row


def test_the_table_has_a_header_and_one_fixed_width_row_per_step(tmp_path):
    # output.rs:246-289, the reference's own row
    with MeasurementLog(str(tmp_path)) as log:
        log.record(dict(mcs=7, cycling=3, quiescent=2, necrotic=1, differentiating=0, apoptotic=5, exposure=0.5,
                        born=9, gone=4, clones=2, lesion=6, vessel=113, perfused=113, sprouts=1, regressed=2,
                        immune=3, killed=4, tissue_radius=12.0, necrotic_radius=1.0 / 3.0, viable_depth=11.666_666))
    lines = (tmp_path / "measurements.csv").read_text().splitlines()
    assert lines[0] == MEASUREMENT_COLUMNS
    assert lines[1] == "7,3,2,1,0,5,0.5000,9,4,2,6,113,113,1,2,3,4,12.0000,0.3333,11.6667"
    assert len(lines[0].split(",")) == len(lines[1].split(","))


def test_a_device_measurement_fills_the_columns_it_has():
    m = dict(mcs=3, cycling=10, quiescent=2, necrotic=4, born=20, gone=1, vessel=0, tissue_radius=5.5,
             necrotic_radius=2.0, viable_depth=3.5)
    assert measurement_row(m) == "3,10,2,4,0,0,0.0000,20,1,1,0,0,0,0,0,0,0,5.5000,2.0000,3.5000"
