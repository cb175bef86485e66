"""Device lattice frames through the `.lm` writer on the GPU
(lmb_lmfile_append_lattice_device / append_sites_device: chunk-order
transpose on the device, copy on the file's stream, compression on the
writer thread): every frame read back equals the lattice's row-major export
(lmb_lattice_get_row_major), on shapes with partial edge chunks and every
slot layout."""
import numpy as np
import pytest

from lattice_microbes_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("X,Y,Z,S,bps", [(20, 18, 35, 8, 1), (9, 7, 5, 4, 4), (17, 33, 16, 16, 4),
                                         (40, 24, 10, 32, 1), (16, 16, 16, 4, 1), (64, 64, 128, 8, 1)])
def test_device_frames_equal_row_major_export(gpu, tmp_path, X, Y, Z, S, bps):
    from lattice_microbes_b200.lmfile import LMFile, LMFileWriter
    from lattice_microbes_b200.solver import Context, Lattice, Model
    spec = configs.random_problem(21, X=X, Y=Y, Z=Z, slots=S, bytes_per_slot=bps, density=1.0, nst=3)
    ctx = Context(0)
    model = Model.from_spec(ctx, spec)
    lat = Lattice(ctx, X, Y, Z, S, bps)
    lat.set_native(spec.lattice, spec.sites)
    p = str(tmp_path / "d.lm")
    w = LMFileWriter(p)
    want = []
    for k in range(4):
        w.append_lattice_device(2, 0.25 * k, lat)
        want.append(lat.get_row_major())
        lat.run(model, 99, 5 * k, 5, check=False)  # the lattice moves on while the frame is written
    w.append_sites_device(2, 1.0, lat)
    sites_now = lat.get_row_major()[1]
    w.close()
    with LMFile(p) as f:
        assert np.array_equal(f.lattice_times(2), [0.0, 0.25, 0.5, 0.75])
        for k, (parts, _) in enumerate(want):
            got = f.lattice(2, k)
            assert got.dtype == (np.uint8 if bps == 1 else np.uint32)
            assert np.array_equal(got, parts)
        assert np.array_equal(f.sites(2, 0), sites_now) and np.array_equal(f.site_times(2), [1.0])
    lat.close()
    model.close()
    ctx.close()
