"""Element set-up on the device (bem3_mesh_pack_dev: init_elem_const and the collocation nodes and
normals of init_boundary_data, d3qd2_setup.c:1139-1186, 1309-1349) against the host set-up, whose
element constants equal the reference's: the geometry records of the three plain configurations
and of a rotated, translated mesh, value for value; an element naming a node outside the table is
refused before anything is read."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_records(p):
    import torch
    from bem3_emf_qd2_b200 import mesh_pack_dev
    rn = torch.from_numpy(np.ascontiguousarray(p.rn, np.float64)).cuda()
    ed = torch.from_numpy(np.ascontiguousarray(p.ed, np.int32)).cuda()
    return mesh_pack_dev(rn, ed).cpu().numpy()


@pytest.mark.parametrize("name", ["sphere384", "twolayer3072", "cone3360"])
def test_device_records_equal_host(cuda_lib, tmp_path, name):
    from bem3_emf_qd2_b200 import MeshArrays, meshgen
    p, _ = meshgen.problem(name, str(tmp_path))
    host = MeshArrays(p).packed()
    dev = _device_records(p)
    assert dev.shape == host.shape
    assert np.array_equal(dev, host), (name, np.abs(dev - host).max())


def test_rotated_mesh(cuda_lib, tmp_path):
    from bem3_emf_qd2_b200 import MeshArrays, meshgen
    from bem3_emf_qd2_b200.dqd2 import load_inputs, problem_from_arrays
    files = meshgen.make_config("cone3360", str(tmp_path))
    p = problem_from_arrays(load_inputs(*files, rot=(1.0, 0.3, 0.0, math.pi / 5, 0.05, -0.02, 0.1)))
    assert np.array_equal(_device_records(p), MeshArrays(p).packed())


def test_node_outside_the_table_is_refused(cuda_lib, tmp_path):
    import torch
    from bem3_emf_qd2_b200 import meshgen, mesh_pack_dev
    p, _ = meshgen.problem("sphere384", str(tmp_path))
    ed = np.ascontiguousarray(p.ed, np.int32).copy()
    ed[7, 2] = p.rn.shape[0] + 5  # past the last node
    rn = torch.from_numpy(np.ascontiguousarray(p.rn, np.float64)).cuda()
    with pytest.raises(RuntimeError):
        mesh_pack_dev(rn, torch.from_numpy(ed).cuda())
    ed[7, 2] = 0  # vertex 0 of a quadrilateral: no node
    with pytest.raises(RuntimeError):
        mesh_pack_dev(rn, torch.from_numpy(ed).cuda())
