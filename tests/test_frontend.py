"""The C++ front end (include/syclfft_b200.hpp) through the reference's own test programs,
restated: tests/native/plugin_tests.cpp (the reference's plugin_tests.cpp: a module with an
incompatible ABI is rejected with plugin_error; runs without a GPU) and
tests/native/frontend_tests.cpp (the reference's sycl_tests.cpp cases; needs a GPU)."""
import os
import subprocess

import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def run(args, env_extra):
    build()
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run([os.path.join(HERE, args[0])] + args[1:], env=env, capture_output=True, text=True,
                          timeout=300)


def test_incompatible_abi_is_a_plugin_error():
    r = run(["plugin_tests", "bad-abi"], {"SYCLFFT_PLUGIN_PATH": os.path.join(HERE, "bad-provider")})
    assert r.returncode == 0, r.stderr


def test_provider_search_path_order():
    r = run(["plugin_tests", "search-path"], {"SYCLFFT_PLUGIN_PATH": "/first::/second"})
    assert r.returncode == 0, r.stderr


def test_module_without_entry_point_is_skipped():
    r = run(["plugin_tests", "no-symbol"], {"SYCLFFT_PLUGIN_PATH": os.path.join(HERE, "nosym-provider")})
    assert r.returncode == 0, r.stderr


def test_extension_argument_checks_need_no_device():
    """Real-transform and strided-layout argument errors (C++ front end) are invalid_argument,
    raised before the provider is loaded or a device is touched."""
    r = run(["plugin_tests", "argument-checks"], {"SYCLFFT_PLUGIN_PATH": ""})
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.gpu
def test_reference_test_program_on_b200():
    r = run(["frontend_tests"], {"SYCLFFT_PLUGIN_PATH": ""})
    assert r.returncode == 0, r.stdout + r.stderr
    assert "front-end tests passed" in r.stdout
