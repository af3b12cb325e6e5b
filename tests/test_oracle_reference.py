"""The CPU oracle reproduces every assertion of the reference's own tests."""


def test_reference_tests_pass_on_the_oracle(oracle):
    failures, checks, report = oracle.selftest()
    assert checks > 100
    assert failures == 0, report
