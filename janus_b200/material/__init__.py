"""Materials (the ``janus.material`` package of the reference)."""
